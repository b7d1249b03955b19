/*
 * matjes_oracle.h -- CPU restatement of the Matjes spin-dynamics hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The tests compare the CUDA path against this
 * library: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg may
 * load it.  The product (matjes_b200) never calls into it.
 *
 * What it restates (paths relative to the Matjes source tree, src/):
 *   - neighbour shells and pair unfolding ........ setup/neighbor_type.f90:78-330
 *   - exchange J term (directed pairs, c_H_J) .... Energy/exchange_Heisenberg_J.f90:23-130
 *   - DMI term and mediator geometry (get_DMI) ... Energy/exchange_Heisenberg_D.f90:23-144, 253-330
 *   - uniaxial anisotropy (c_H_ani) .............. Energy/anisotropy_heisenberg.f90:148-292
 *   - Zeeman ("BM" term, c_zeeman) ............... Energy/zeeman.f90:30-86
 *   - 1e-10 relative coefficient drop ............ Energy/setH_util.f90:10-36
 *   - field B = -(H m + H^T m) - Hz^T b, -2 H_fft  Hamiltonian_type/hamiltonian_collection.f90:433-454
 *   - per-site / total energy .................... Hamiltonian_type/ham_base.f90:181-260,
 *                                                  Hamiltonian_type/fft_ham_base.f90:247-267
 *   - dipolar K tensor, N_rep/padding rule ....... Energy/dipolar_magnetic.f90:58-177, 275-308,
 *                                                  Hamiltonian_type/fft_ham_base.f90:191-245,
 *                                                  Hamiltonian_type/fft_ham_internal.f90:26-123
 *   - explicit O(N^2) dipolar check path ......... Energy/dipolar_magnetic.f90:181-273
 *   - LLG right-hand side ........................ solvers/propagator.f90:13-58
 *   - projected Euler update ..................... solvers/solver.f90:97-118
 *   - stage loop, Butcher factors, noise draw .... dynamics/spindynamics.f90:260-323,
 *                                                  solvers/solver_order.f90:14-127
 *   - thermal torque (langevin_bath) ............. dynamics/BTeff_sd.f90:18-45
 *   - noise sigma = sqrt(alpha kT hbar / dt) ..... dynamics/spindynamics.f90:268-272
 *   - constants .................................. fixed-parameters/constant.f90:11-32
 *   - Metropolis move, acceptance ................ Metropolis-MC/MCstep.f90:37-89
 *   - GNEB path relaxation (VPO) ................. GNEB/gneb_utils.f90:19-240, GNEB/path.f90:10-29,
 *                                                  GNEB/tangent.f90:89-180, utilities/rotation.f90
 *   - random site, proposals, cone update ........ Metropolis-MC/choosespin.f90:13-21,
 *                                                  Metropolis-MC/track_value.f90:84-160,
 *                                                  Metropolis-MC/relaxationtype.f90:15-70,
 *                                                  paratemp-MC/sampling.f90:9-62
 *
 * SIB is absent from the reference (solvers/solver_commun.f90:97-108 has it
 * commented out); the SIB here restates the published semi-implicit scheme of
 * Mentink, Tretyakov, Fasolino, Katsnelson, Rasing, J. Phys.: Condens. Matter
 * 22, 176001 (2010) on Matjes' field, units and Landau-Lifshitz form.
 *
 * Pinning: the Euler path (precession sense, projection, Zeeman and exchange
 * energy per site) is pinned against the reference's own golden file
 * tests/serial/isolated_spin_precession/Euler/REF (committed as a fixture).
 * The remaining terms are pinned by analytic known-answer tests and by the
 * independent explicit dipolar sum; the reference itself cannot be compiled
 * here (no Fortran compiler), so field parity beyond those is "partially
 * pinned".
 *
 * Layout: AoS, m[3*site + comp], site = cell*Nmag + imag,
 * cell = x + Lx*(y + Ly*z) (Matjes index_m_1 with x fastest, 0-based).
 */
#ifndef MATJES_ORACLE_H
#define MATJES_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXAT 16
#define ORC_MAXTERM 32

/* physical constants, fixed-parameters/constant.f90:11-32 */
#define ORC_KB 0.000086173324
#define ORC_PI 3.14159265358979323846
#define ORC_MUB 0.0000578838180661
#define ORC_HBAR 0.658211928
#define ORC_DIP_PREF 6.745817653234234066975e-7 /* Energy/dipolar_magnetic.f90:41 */

typedef struct {
    int L[3];
    int periodic[3];
    double areal[3][3];        /* rows: lattice vectors in nm (alat applied) */
    int natom;
    double frac[ORC_MAXAT][3]; /* fractional coordinates of the cell atoms */
    int attype[ORC_MAXAT];     /* atom type id (1-based, as in the input deck) */
    double moment[ORC_MAXAT];  /* magnetic moment in mu_B; > 0 means magnetic */
} orc_lattice;

typedef struct { int t1, t2, shell; double J; } orc_J;           /* magnetic_J  t1 t2 shell J */
typedef struct { int t1, t2, tmed, shell; double D; } orc_D;     /* magnetic_D  t1 t2 tmed shell D */
typedef struct { int type; double axis[3]; double K; } orc_K;    /* magnetic_anisotropy */

typedef struct {
    orc_lattice lat;
    int nJ; orc_J J[ORC_MAXTERM];
    int nD; orc_D D[ORC_MAXTERM];
    int nK; orc_K K[ORC_MAXTERM];
    double c_H_J, c_H_D, c_H_ani, c_zeeman;   /* -1, -1, +1, -1 in the reference */
    double B_ext[3];                          /* H_ext in Tesla */
    int zeeman_on;
    int dip_on;                               /* 1: the reference's grid rule; 2: every axis
                                                 longer than one cell zero-padded to 2 L */
    int dip_period_cut[3];                    /* mag_dip_period_cut, default 1 1 1 */
} orc_input;

typedef struct orc_model orc_model;

enum { ORC_EULER = 1, ORC_HEUN_MATJES = 2, ORC_SIB = 3 };
enum { ORC_NOISE_OFF = 0, ORC_NOISE_PHILOX = 1, ORC_NOISE_INJECT = 2 };

void orc_input_defaults(orc_input* in);

/* Build the Hamiltonian (COO -> CSR) the way set_Hamiltonians does. 0 on success. */
int orc_model_build(const orc_input* in, orc_model** out);
void orc_model_free(orc_model* m);

int64_t orc_nsites(const orc_model* m);
int orc_nmag(const orc_model* m);
int64_t orc_mm_nnz(const orc_model* m);
/* COO export of the combined MM matrix (0-based rows/cols, 3N x 3N). */
int orc_mm_coo(const orc_model* m, int64_t cap, int64_t* rows, int64_t* cols, double* vals);
/* Per-site Zeeman field b (Tesla) override, AoS 3*Ncell. NULL restores the uniform H_ext. */
int orc_set_bfield(orc_model* m, const double* b_cell);
/* Dipolar grid N_rep (reference padding rule). */
void orc_dip_nrep(const orc_model* m, int nrep[3]);

/* Effective field B = -dE/dm (eV) and per-site energy (eV, may be NULL).
 * e_site follows energy_distrib: per term left-assigned, dipolar doubled. */
void orc_field(const orc_model* m, const double* mvec, double* B, double* e_site);
/* Total energy H%energy(lat) (eV, not divided by N). */
double orc_energy(const orc_model* m, const double* mvec);
/* Minimisation drivers (solvers/minimize.F90:57-166 and :169-258), see matjes_oracle.c. */
int orc_minimize_vpo(const orc_model* M, double* m, double dt, double mass, double conv_torque, int64_t niter,
                     int64_t* iters, double* max_torque);
int orc_minimize_infdamp(const orc_model* M, double* m, double conv_torque, int64_t niter, const int colors[3],
                         int64_t* iters, double* max_torque);
/* GNEB minimum-energy path of nim images img (nim x N x 3, AoS per image; the
 * end images stay fixed), single-atom models: find_path (GNEB/gneb_utils.f90:
 * 19-240), with the climbing image when climb != 0 (the first image of highest
 * energy, chosen again each iteration; its force F - 2 tau (F.tau), no spring;
 * ci_out, may be NULL, the last one, 0-based, or -1).  The reference's
 * truncation of velocity and force components below 1e-50 of their maximum
 * (vector_utils/precision.f90) is left out: it cannot change a double result
 * here.  Each iteration moves the interior images
 * by velocity Verlet on the unit sphere (m + v dt + F dt^2 / 2 mass,
 * normalised), parallel-transports velocity and old force by the rotation of
 * each spin's move (utilities/rotation.f90 rotate), recomputes the projected
 * fields, energies, path length (path.f90 the_path) and GNEB forces (force
 * perpendicular to the energy-weighted tangent, tangent.f90:89-124, plus the
 * spring force k (l_{i+1} + l_{i-1} - 2 l_i) along it), and projects the
 * velocity on the force (VPO); it stops when max |F| < ftol.  rx, ene (minus
 * the initial (en_zero 'I'), final ('F') or no ('N') image energy) and dene =
 * -F.tau_single per image as en_path.out holds them. */
int orc_gneb_find_path(const orc_model* M, double* img, int nim, double spring, double dt, double mass, double ftol,
                       int64_t itrmax, int en_zero, int climb, double* rx, double* ene, double* dene, int64_t* iters,
                       double* fchk_out, int* ci_out);
/* OpenMP threads of the parallel loops (n <= 0: all processors). */
void orc_set_threads(int n);
/* Metropolis Monte Carlo.  proposal: 0 sphereft cone, 1 Ising flip,
 * 2 under-relaxation, 3 over-relaxation.  The uniforms are Philox4x32-10 words
 * under key `seed`, each turned into (w + 0.5) 2^-32. */
typedef struct {
    double temperature, cone;
    int proposal, adapt_cone;
    uint64_t seed;
    uint32_t stream_id, sweep0;
    int64_t accepted_total, proposed_total;
} orc_mc;
/* Sweeps colour by colour (single-atom models): colours 0 .. ncolours-1 in
 * turn (site_colour[i] the colour of site i), each colour's sites in index
 * order; site i of sweep t draws counter (i, t, stream, 0x4D43): words 0, 1
 * the proposal, 2 the test.  After each sweep E_out[k] = H%energy, M_out[3k..]
 * = summed spins; the cone update of an adaptive cone proposal runs once per
 * sweep with step 1e-4 N. */
int orc_mc_sweeps(const orc_model* M, double* m, orc_mc* p, int nsweeps, const int* site_colour, int ncolours,
                  double* E_out, double* M_out, int64_t* accepted);
/* The reference's order: N moves per sweep at sites chosen by choose_spin
 * (1 + INT(u (N-1)), so the last site never moves), move t of sweep k drawing
 * counter (t, k, stream, 0x52534D43): word 0 the site, 1, 2 the proposal, 3
 * the test; the cone update before each cone proposal; E_out and M_out the
 * incrementally tracked totals of track_val after each sweep. */
int orc_mc_random(const orc_model* M, double* m, orc_mc* p, int nsweeps, double* E_out, double* M_out,
                  int64_t* accepted);
/* Field contributions split: MM only, Zeeman only, dipolar only (for tests). */
void orc_field_terms(const orc_model* m, const double* mvec, double* B_mm, double* B_zee, double* B_dip);
/* Route of the model's dipolar convolution: 1 = the direct circular sum,
 * 0 = the FFT route where the grid is a power of two in every axis (default). */
void orc_dip_direct(orc_model* m, int direct);
/* Explicit O(N^2) dipolar field (get_dipolar, mag_dip_fft F). */
void orc_dipolar_explicit_field(const orc_model* m, const double* mvec, double* B);

/* The table-driven log(u) and sin/cos(2 pi u) of the Box-Muller draw for
 * u = (w + 1/2) 2^-32 of 32-bit words w. */
void orc_tab_eval(const uint32_t* w, int64_t n, double* lg, double* s, double* c);
/* Raw Philox4x32-10 block (for the Random123 known-answer vectors). */
void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Philox4x32-10 N(0,1) triples, identical counter layout to the product. */
void orc_philox_normals(uint64_t seed, uint32_t step, uint32_t stream, int64_t site0,
                        int64_t nsite, double* out /* AoS 3*nsite */);

typedef struct {
    int integrator;      /* ORC_EULER / ORC_HEUN_MATJES / ORC_SIB */
    double timestep;     /* fs */
    double alpha;        /* damping */
    double temperature;  /* K */
    int noise;           /* ORC_NOISE_* */
    uint64_t seed;
    uint32_t stream;     /* replica id folded into the Philox counter */
    uint32_t step0;      /* global step index of the first step */
    const double* inject;/* N(0,1) buffer, layout [nbuf][3][N] */
    int inject_nbuf;
    int energy_before;   /* E_step[k]: 0 = energy after step k (an extra field pass,
                            spindynamics.f90:323); 1 = energy of the state step k
                            starts from, summed in the first stage's field pass */
} orc_dyn;

/* Advance nsteps; m updated in place; E_step[k] as orc_dyn.energy_before says (may be NULL). */
int orc_run(const orc_model* m, const orc_dyn* d, double* mvec, int nsteps, double* E_step);

/* Rotation sense helpers for tests */
void orc_llg_torque(const double* B, double alpha, const double* m, double* D, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
