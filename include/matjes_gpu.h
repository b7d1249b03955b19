/*
 * matjes_gpu.h -- C ABI of the B200-native Matjes spin-dynamics hot path.
 *
 * Plain C: pointers, fixed-width integers and doubles only; no CUDA or torch
 * types in any signature (a stream is passed as `void*` holding a
 * cudaStream_t, NULL = legacy default stream).  Every call returns an
 * mj_status; mj_last_error() gives the message of the last failure on the
 * calling thread.  Nothing aborts.
 *
 * Physical conventions are Matjes' own (src/ paths of the Matjes tree):
 *   energies and fields in eV (B_eff = -dE/dm), applied field in Tesla,
 *   time in fs, lengths in nm, hbar = 0.658211928 eV fs
 *   (fixed-parameters/constant.f90:28), the Landau-Lifshitz form of
 *   solvers/propagator.f90:13-58.
 *
 * Host arrays use the reference layout (AoS, m[3*site+comp], site =
 * cell*Nmag + imag, cell = x + Lx*(y + Ly*z));  device arrays are SoA
 * (x[N], y[N], z[N] with one base pointer of 3N doubles).
 */
#ifndef MATJES_GPU_H
#define MATJES_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t mj_status;
enum {
    MJ_OK = 0,
    MJ_ERR_ARG = 1,         /* bad argument / size */
    MJ_ERR_OOM = 2,         /* device or host allocation failed */
    MJ_ERR_CUDA = 3,        /* CUDA runtime / cuFFT error */
    MJ_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
    MJ_ERR_NAN = 5,         /* non-finite value detected in the state */
    MJ_ERR_UNSUPPORTED = 6, /* input outside what the kernels implement */
    MJ_ERR_GEOMETRY = 7     /* shell / DMI geometry could not be built */
};

enum { MJ_EULER = 1, MJ_HEUN_MATJES = 2, MJ_SIB = 3 };
enum { MJ_NOISE_OFF = 0, MJ_NOISE_PHILOX = 1, MJ_NOISE_INJECT = 2 };

#define MJ_MAX_ATOMS 16

/* Lattice and cell: IO-input/rw_lattice.f90:28-80 (Periodic_log, alat,
 * lattice, Nsize) and IO-input/rw_cell.f90:5-31 (atomtypes / atoms). */
typedef struct {
    int32_t L[3];            /* Nsize */
    int32_t periodic[3];     /* Periodic_log */
    double areal[3][3];      /* lattice vectors as rows, in nm (alat applied) */
    int32_t natom;
    double frac[MJ_MAX_ATOMS][3];  /* fractional atom positions */
    int32_t attype[MJ_MAX_ATOMS];  /* atom type id (1-based) */
    double moment[MJ_MAX_ATOMS];   /* magnetic moment in mu_B, > 0 = magnetic */
} mj_lattice_desc;

/* magnetic_J  t1 t2 shell J  (Energy/exchange_Heisenberg_J.f90:18-130) */
typedef struct { int32_t t1, t2, shell; double value; } mj_exchange_term;
/* magnetic_D  t1 t2 mediator shell D  (Energy/exchange_Heisenberg_D.f90:11-144) */
typedef struct { int32_t t1, t2, tmed, shell; double value; } mj_dmi_term;
/* magnetic_anisotropy  type  ex ey ez  K  (Energy/anisotropy_heisenberg.f90:148-292) */
typedef struct { int32_t type; double axis[3]; double value; } mj_aniso_term;

typedef struct {
    int32_t nJ; const mj_exchange_term* J;
    int32_t nD; const mj_dmi_term* D;
    int32_t nK; const mj_aniso_term* K;
    double c_H_J, c_H_D, c_H_ani, c_zeeman; /* reference defaults: -1, -1, +1, -1 */
    double B_ext[3];                        /* H_ext (Tesla) */
    int32_t zeeman_on;                      /* enable_H; also on when |H_ext| >= 1e-8 */
    int32_t dip_on;                         /* mag_dip_use (FFT route): 1 = the reference's grid
                                               (Hamiltonian_type/fft_ham_base.f90:204-214: open axes
                                               doubled, periodic axes kept, images folded in); 2 = every
                                               axis longer than one cell zero-padded to 2 L (a linear
                                               convolution, images summed over -cut..cut for every pair
                                               as in the explicit route dipolar_magnetic.f90:181-273;
                                               no counterpart flag in the reference) */
    int32_t dip_period_cut[3];              /* mag_dip_period_cut, default 1 1 1 */
} mj_hamiltonian_desc;

typedef struct {
    int32_t integrator;   /* MJ_EULER, MJ_HEUN_MATJES, MJ_SIB */
    double timestep;      /* fs (the deck's `timestep`) */
    double alpha;         /* damping */
    double temperature;   /* K */
    int32_t noise;        /* MJ_NOISE_* */
    uint64_t seed;        /* Philox key */
    uint32_t stream_id;   /* replica id folded into the Philox counter */
    uint32_t step0;       /* global index of the first step (Philox counter / inject slot) */
    const double* inject; /* device N(0,1) buffer, layout [nbuf][3][N] (MJ_NOISE_INJECT) */
    int32_t inject_nbuf;
    int32_t energy_mode;  /* MJ_ENERGY_AFTER (reference: E after each step, one extra
                             field pass per call) or MJ_ENERGY_BEFORE (E of the state
                             entering each step, fused into the first pass, no extra pass) */
} mj_dyn_params;

enum { MJ_ENERGY_AFTER = 0, MJ_ENERGY_BEFORE = 1 };

typedef struct mj_plan mj_plan;
typedef struct mj_state mj_state;

/* ---- errors ---------------------------------------------------------- */
/* Message of the last failing call on this thread (never NULL). */
const char* mj_last_error(void);
/* Library version string. */
const char* mj_version(void);

/* ---- plans (Hamiltonian + lattice, device resident) ------------------- */
/* Replaces the Hamiltonian set-up path setup/setup-simu.f90:104-110 ->
 * Energy/set_Hamiltonians.f90:9-180 -> Hamiltonian_type/ham_cusparse.f90:134-153
 * -> cuda_H_init (Hamiltonian_type/cuda_H.cu:45-133), and for the dipolar term
 * Energy/set_fft_Hamiltonians.f90:8-79 -> cuda_fft_init / set_cuda_fft_plan /
 * cuda_fft_set_operator (Hamiltonian_type/cuda_fft.cpp:10-143).  Shells are
 * rebuilt on the host exactly like setup/neighbor_type.f90:78-330; single-atom
 * cells become a fused stencil, multi-atom cells an ELL matrix. */
mj_status mj_plan_create(const mj_lattice_desc* lat, const mj_hamiltonian_desc* ham,
                         int32_t device, mj_plan** out);
/* Replaces cuda_H_init (Hamiltonian_type/cuda_H.cu:45-133) for a Hamiltonian
 * handed over as COO triplets (the reference passes 1-based rows/cols,
 * Hamiltonian_type/ham_coo.f90:158-196; `base` is 0 or 1).  The triplets are
 * the combined "MM" matrix H (3N x 3N); zeeman[s] is the "BM" coefficient
 * mu0*muB*c_zeeman*mu_s of site s and b_cell the applied field per cell.  The
 * field is B = -(H + H^T) m - zeeman*b. */
mj_status mj_plan_from_coo(int64_t nsites, int64_t nnz, const int64_t* rows, const int64_t* cols,
                           const double* vals, int32_t base, const double* zeeman,
                           const double* b_cell, int32_t device, mj_plan** out);
/* Replaces cuda_H_destroy / cuda_fft destroy (cuda_H.cu:315-344, cuda_fft.cpp:145-180). */
mj_status mj_plan_destroy(mj_plan* plan);
/* Number of spin sites N (= Ncell * Nmag). */
mj_status mj_plan_nsites(const mj_plan* plan, int64_t* n);
/* Stencil introspection: number of neighbour offsets (0 for ELL plans). */
mj_status mj_plan_noffsets(const mj_plan* plan, int32_t* n);
/* Kernel variant of a stencil plan: -1 = generic per-offset kernel; 0..5 =
 * shared-memory tiled kernel with 32 x (threads-in-y * sites-per-thread)
 * tiles of 4x4, 8x4, 8x2, then 4x4, 8x2, 4x2 compiled for 6, 4, 8 resident
 * blocks per SM (fewer registers).  Tiled variants exist for the square (NN,
 * NN+NNN) and triangular (NN, three shells) offset sets; MJ_ERR_UNSUPPORTED
 * otherwise.  No counterpart in the reference (its SpMV has no tiling). */
mj_status mj_plan_set_variant(mj_plan* plan, int32_t variant);
/* Current variant (-1 generic) and the matched compile-time shape id (0 none). */
mj_status mj_plan_get_variant(const mj_plan* plan, int32_t* variant, int32_t* shape);
/* Halo staging of the tiled kernels (one tile per block either way): enable = 1
 * (default) stages tile + halo with one TMA bulk-tensor copy while the block
 * computes its thermal draw, then rewrites the halo cells across a periodic
 * edge with plain loads (the copy fills cells outside the lattice with zeros,
 * the open boundary); 0 = plain loads with the periodic wrap per element.
 * Lattices with an odd Lx or a spin array not 16-byte aligned use plain loads. */
mj_status mj_plan_set_tma(mj_plan* plan, int32_t enable);
/* SIB steps of tiled plans without the dipolar term: enable = 1 runs
 * predictor and corrector in one launch (k_sib_fused: blocks take tiles from a
 * work counter, a corrector tile starts as soon as the predictor rows its
 * stencil reaches are done); 0 (default) = two launches.  The results are the
 * same bit for bit.  No counterpart in the reference. */
mj_status mj_plan_set_fused(mj_plan* plan, int32_t enable);
/* Kernel options of a stencil plan (none changes a result, every one only how
 * it is computed; no counterpart in the reference):
 *   MJ_OPT_TMA, MJ_OPT_FUSED   as mj_plan_set_tma / mj_plan_set_fused;
 *   MJ_OPT_PDL (default 1)     tiled passes launched as programmatic dependents
 *                              of the kernel before them: the next pass launches
 *                              while this one's last blocks run, and a predictor
 *                              computes its thermal draw before it waits for the
 *                              previous kernel's results;
 *   MJ_OPT_STORE_DRAW (default 1)  SIB with Philox noise: the predictor stores
 *                              its draw for the corrector (24 B per site written
 *                              and read back) instead of the corrector drawing
 *                              it again (the same numbers either way);
 *   MJ_OPT_HOST_STRIPES (0 = default 4, at most 64)  stripes of tile rows that
 *                              mj_step_host cuts a one-step call with pinned
 *                              host spins into (fewer when the lattice has
 *                              fewer than 5 tile rows per stripe);
 *   MJ_OPT_BLOCKS_PER_SM (0 = default: no cap, else 4..32)  at most this many
 *                              blocks of a tiled pass resident per SM (each
 *                              launch asks for enough shared memory), so that
 *                              the tiles of a lattice fill the last wave of
 *                              the GPU better;
 *   MJ_OPT_DIP_ZCONV (default 1)  FFT dipolar term with a z grid of a power
 *                              of two up to 32: the z transforms and the
 *                              product with K_F as one kernel (0: cuFFT z
 *                              transforms and a separate product);
 *   MJ_OPT_HOST_ZEROCOPY (default 1)  striped mj_step_host with a mapped pinned
 *                              buffer: kernels write the stepped spins into it
 *                              directly (0: device transposes and copies). */
enum {
    MJ_OPT_TMA = 0,
    MJ_OPT_FUSED = 1,
    MJ_OPT_PDL = 2,
    MJ_OPT_STORE_DRAW = 3,
    MJ_OPT_HOST_STRIPES = 4,
    MJ_OPT_BLOCKS_PER_SM = 5,
    MJ_OPT_DIP_ZCONV = 6,
    MJ_OPT_HOST_ZEROCOPY = 7
};
mj_status mj_plan_set_option(mj_plan* plan, int32_t option, int32_t value);
/* Autotuner: times `steps` steps of `p` for every kernel configuration of the
 * plan on a scratch copy of the device spins m_dev_soa (left untouched), keeps
 * the fastest and returns its variant in *best (and its staging in *best_tma,
 * may be NULL).  ms_per_step (13 doubles, may be NULL): [0] generic kernel,
 * [1+v] tiled variant v with plain loads, [7+v] with TMA; negative = not
 * available.  Synchronous. */
mj_status mj_plan_autotune(mj_plan* plan, const double* m_dev_soa, const mj_dyn_params* p, int32_t steps,
                           int32_t* best, int32_t* best_tma, double* ms_per_step);
/* Device status word of the plan's kernels (synchronises, then clears it):
 * MJ_ERR_TIMEOUT when a bounded device wait gave up since the last check (the
 * results of that launch are invalid), else MJ_ERR_NAN when a time step wrote a
 * non-finite spin component (the state is invalid from that step on).  The
 * asynchronous step calls (mj_step, mj_step_dev, mj_graph_run) leave the report
 * to this call; mj_step_host and mj_gneb_path return it themselves.  The
 * reference has no such report: its only check is the energy-increase warning of
 * dynamics/spindynamics.f90:376-381. */
mj_status mj_plan_check_status(mj_plan* plan);
/* Self-test of the failure path of the bounded device waits (no counterpart in
 * the reference): one block arms an mbarrier for 16 bytes that no copy delivers
 * (nothing is issued, so nothing is in flight), polls it `polls` times (1 ..
 * 65536) through the same bounded wait as the tiled kernels' TMA staging, gives
 * up and records the timeout in the plan's status word as they do; the next
 * mj_plan_check_status returns MJ_ERR_TIMEOUT and clears it.  Asynchronous on
 * `stream`. */
mj_status mj_plan_selftest_timeout(mj_plan* plan, uint32_t polls, void* stream);
/* Per-site applied field map (Tesla, host AoS 3*Ncell; NULL = uniform H_ext):
 * the Bfield_init.dat input read by initialization/orders_initialize.f90:28. */
mj_status mj_plan_set_bfield(mj_plan* plan, const double* b_cell_host);
/* Same, from a device SoA buffer (3*Ncell doubles, copied). */
mj_status mj_plan_set_bfield_device(mj_plan* plan, const double* b_cell_dev_soa, void* stream);

/* Host-only (touches no GPU): the fused stencil a single-atom deck compiles to,
 * i.e. the couplings Energy/set_Hamiltonians.f90:9-180 would hand to
 * cuda_H_init, folded per neighbour offset: B_i = sum_o W_o m_{i+o} + W0 m_i
 * + zc b_i with W_o = -(T_o + T_{-o}^T).  offsets: 3*cap ints, W: 9*cap doubles
 * (row-major), W0: 9 doubles.  MJ_ERR_UNSUPPORTED for multi-atom cells. */
mj_status mj_stencil_describe(const mj_lattice_desc* lat, const mj_hamiltonian_desc* ham, int32_t cap,
                              int32_t* n_off, int32_t* offsets, double* W, double* W0, double* zc);

/* ---- states (spin field, device resident SoA) ------------------------- */
/* Replaces cuda_fvec_init / cuda_fvec_alloccopy (cuda_H_vec.cu:11-43). */
mj_status mj_state_create(const mj_plan* plan, mj_state** out);
mj_status mj_state_destroy(mj_state* st);
/* Host AoS -> device SoA (cuda_fvec_set, cuda_H_vec.cu:60-73). */
mj_status mj_state_upload(mj_state* st, const double* m_host_aos, void* stream);
/* Device SoA -> host AoS (cuda_fvec_get, cuda_H_vec.cu:75-88). */
mj_status mj_state_download(const mj_state* st, double* m_host_aos, void* stream);
/* Device pointer of the SoA spin field (3N doubles: x block, y block, z block). */
mj_status mj_state_device_ptr(const mj_state* st, double** m_dev_soa);

/* ---- field and energy ------------------------------------------------- */
/* B_eff = -dE/dm: hamiltonian%get_eff_field (Hamiltonian_type/hamiltonian_collection.f90:433-454,
 * reached from dynamics/spindynamics.f90:298).  Device SoA output (3N); e_site
 * (device, N, may be NULL) is the per-site energy of energy_distrib
 * (hamiltonian_collection.f90:332-363). */
mj_status mj_field(mj_plan* plan, const mj_state* st, double* B_dev_soa, double* e_site_dev, void* stream);
/* Same on caller-owned device SoA spins (torch tensors). */
mj_status mj_field_dev(mj_plan* plan, const double* m_dev_soa, double* B_dev_soa, double* e_site_dev, void* stream);
/* hamiltonian%energy (hamiltonian_collection.f90:390-400): total energy in eV,
 * synchronous, written to *E_host. */
mj_status mj_energy(mj_plan* plan, const mj_state* st, double* E_host);
/* Total energy (as mj_energy) of device spins m_dev_soa (3N doubles, SoA) into
 * *E_dev (one device double), on `stream`, without allocating anything.  No
 * counterpart in the reference.  It is meant for callers that cannot call
 * cudaMalloc when they evaluate the energy: a host code whose GPU memory is
 * handed out by its own pool or capped by its job scheduler once set up, or a
 * driver that must not allocate inside its time loop.  Its scratch (one
 * partial sum per thread block and a ticket counter) is a fixed static device
 * array of MJ_NOALLOC_MAX_BLOCKS doubles (512 KiB) that every GPU loading the
 * library holds until the process exits.  The limit is on thread blocks, one
 * per 32 x 8 tile of a layer for stencil plans (ceil(Lx/32) * ceil(Ly/8) * Lz
 * <= 65536) and one per 256 sites for ELL plans (ceil(N/256) <= 65536); a
 * lattice over it is rejected with MJ_ERR_ARG.  2^24 sites is an upper bound,
 * not a guarantee: 4095 x 4097 (2^24 - 1 sites) already needs 128 x 513 =
 * 65664 blocks.  Plans with the FFT dipolar term are rejected with
 * MJ_ERR_UNSUPPORTED.  The first call on a device looks
 * up the array's device address: make that first call before any stream
 * capture.  All calls share the one array and each leaves its partial sums in
 * it: calls that overlap on the GPU (different streams or host threads) race,
 * so serialise them. */
#define MJ_NOALLOC_MAX_BLOCKS 65536
mj_status mj_energy_noalloc(const mj_plan* plan, const double* m_dev_soa, double* E_dev, void* stream);
/* Host-array convenience form of get_eff_field (reference AoS layout); it
 * uploads m, evaluates, downloads B and e_site (may be NULL); synchronous. */
mj_status mj_field_host(mj_plan* plan, const double* m_host_aos, double* B_host_aos, double* e_site_host);

/* ---- dynamics ----------------------------------------------------------- */
/* nsteps LLG time steps in place: the loop body dynamics/spindynamics.f90:260-323
 * (stage loop 282-313, thermal field 268-272, energy 323).  E_dev (device,
 * nsteps doubles, may be NULL) receives H%energy after each step. */
mj_status mj_step(mj_plan* plan, mj_state* st, const mj_dyn_params* p, int32_t nsteps,
                  double* E_dev, void* stream);
/* Same on caller-owned device SoA spins. */
mj_status mj_step_dev(mj_plan* plan, double* m_dev_soa, const mj_dyn_params* p, int32_t nsteps,
                      double* E_dev, void* stream);
/* Host-array convenience: upload m, run nsteps, download m and E (host, may be NULL).
 * Synchronous; returns MJ_ERR_NAN when a step wrote a non-finite spin component
 * (MJ_ERR_TIMEOUT when a bounded wait gave up), as mj_plan_check_status. */
mj_status mj_step_host(mj_plan* plan, double* m_host_aos, const mj_dyn_params* p, int32_t nsteps,
                       double* E_host);
/* The step loop captured once as a CUDA graph of `nsteps` steps and replayed
 * `nreplay` times (steps advance p->step0 by nsteps per replay). */
mj_status mj_graph_run(mj_plan* plan, mj_state* st, const mj_dyn_params* p, int32_t nsteps,
                       int32_t nreplay, double* E_dev, void* stream);

/* Per-kernel device timing of a plan (CUDA events around every kernel the plan
 * launches), the evidence behind the achieved-bandwidth figures; no
 * counterpart in the reference, which only times the whole dynamics with
 * cpu_time (dynamics/spindynamics.f90:118,456-457).  enable != 0 clears the
 * accumulators and starts recording; mj_profile_read synchronises and returns
 * up to `cap` kernels: names (32 chars each), total ms and launch counts. */
mj_status mj_profile_enable(mj_plan* plan, int32_t enable);
mj_status mj_profile_read(mj_plan* plan, int32_t cap, char* names, double* total_ms, int64_t* launches,
                          int32_t* n);

/* Thermal helpers: reference temperature estimator T = sum|m x B|^2 / (2 kB sum m.B)
 * (dynamics/measure_temp.f90:21-43), synchronous. */
mj_status mj_measure_temperature(mj_plan* plan, const mj_state* st, double* T_host);
/* Philox N(0,1) triples exactly as the thermal kernels draw them (device SoA [3][n]). */
mj_status mj_philox_normals(uint64_t seed, uint32_t step, uint32_t stream_id, int64_t n,
                            double* out_dev_soa, void* stream);

/* ---- energy minimisation (solvers/minimize.F90) --------------------------- */
/* min_input of IO-input/minimize_io.f90:6-12: `timestep`, `masse`,
 * `convergence_criteria`; the host looks at the convergence flag every
 * `check_every` iterations (the reference prints every `min_Efreq`). */
typedef struct {
    double timestep;
    double mass;
    double conv_torque;
    int32_t check_every;
} mj_min_params;
/* minimize_run (solvers/minimize.F90:57-166) on the device spins, in place:
 * velocity projection on the damping force F = B - (m.B) m, the first predictor
 * unnormalised and later moves keeping each spin's norm, as in the reference.
 * Stops after max_iter iterations or when the largest |F| drops below
 * conv_torque; returns the iterations run and that torque.  Any plan. */
mj_status mj_minimize(mj_plan* plan, double* m_dev_soa, const mj_min_params* p, int64_t max_iter,
                      int64_t* iterations, double* max_torque, void* stream);
/* minimize_infdamp_run (solvers/minimize.F90:169-258): every spin turned onto
 * its normalised local field; the sites are visited colour by colour (colours
 * (x mod cx) + cx((y mod cy) + cy(z mod cz)) returned in colors[3], chosen so
 * that no coupling joins two sites of one colour) instead of in site order.
 * The torque is the largest component of m x B^.  Single-atom stencil plans
 * without the dipolar term; MJ_ERR_ARG when a site's field is below 1e-8 (the
 * reference stops there). */
mj_status mj_minimize_infdamp(mj_plan* plan, double* m_dev_soa, const mj_min_params* p, int64_t max_iter,
                              int64_t* iterations, double* max_torque, int32_t* colors, void* stream);

/* ---- Metropolis Monte Carlo (Metropolis-MC/MCstep.f90) ------------------- */
/* Proposals of Metropolis-MC/track_value.f90: sample_sphere (sphereft of
 * paratemp-MC/sampling.f90:9-62, a uniform direction in the cone about the old
 * spin), sample_ising (the flip), sample_underrelax / sample_overrelax
 * (Metropolis-MC/relaxationtype.f90, from the site's effective field).  The
 * reference's equi_samp draws the same uniform-in-the-cone distribution as
 * sphereft by rejection; a caller maps it to MJ_MC_CONE. */
enum { MJ_MC_CONE = 0, MJ_MC_ISING = 1, MJ_MC_UNDERRELAX = 2, MJ_MC_OVERRELAX = 3 };
typedef struct {
    double temperature;      /* K */
    double cone;             /* half-angle of the proposal cone (rad); updated when adapt_cone */
    int32_t proposal;        /* MJ_MC_* */
    int32_t adapt_cone;      /* 1: the reference's rate-driven cone update (track_value.f90 cone_update) */
    uint64_t seed;           /* Philox key */
    uint32_t stream_id;      /* replica id folded into the Philox counter */
    uint32_t sweep0;         /* index of the next sweep (advanced by each call) */
    int64_t accepted_total;  /* running counts of accepted and proposed moves */
    int64_t proposed_total;
    uint32_t round0;         /* index of the next parallel-tempering round (mj_batch_mc) */
    int32_t track_totals;    /* mj_mc_sweeps: 1 = E_dev / M_dev are the totals of the call's start
                                updated by every accepted move (track_val's E_total and
                                Magnetization), 0 = recomputed after every sweep */
} mj_mc_params;
/* nsweeps Metropolis sweeps on the device spins, in place: every site moved
 * once per sweep, colour by colour in a colouring where no coupling joins two
 * sites of one colour.  colors[4] returns it: {q, b, c, 1} for the linear
 * colour (x + b y + c z) mod q, moved k = 0 .. q-1 in turn, or {cx, cy, cz, 0}
 * for the product colour (x mod cx, y mod cy, z mod cz), moved with x mod cx
 * fastest; the one with fewer colours is chosen.  Each move makes the proposal
 * and the acceptance test of
 * MCstep.f90:75-89 on the single-site energy change.  The reference moves
 * randomly chosen sites (choose_spin.f90) with a sequential generator; here
 * the uniforms are Philox draws, counter (site, sweep, stream_id, 0x4D43).
 * E_dev (nsweeps doubles) and M_dev (3 nsweeps) receive the energy and the
 * summed spins after each sweep (either may be NULL); *accepted the accepted
 * moves of the call.  Single-atom stencil plans without the dipolar term
 * (MJ_ERR_UNSUPPORTED otherwise, and when neither a linear colouring of at
 * most 16 colours nor a product one of at most 4 x 4 x 4 fits the stencil and
 * the periodic sizes).  The adaptive cone (sample_sphere) is updated once per
 * sweep by 1e-4 per move of the sweep from the running acceptance rate. */
mj_status mj_mc_sweeps(mj_plan* plan, double* m_dev_soa, mj_mc_params* p, int32_t nsweeps, double* E_dev,
                       double* M_dev, int64_t* accepted, int32_t* colors, void* stream);

/* ---- reverse mode (adjoint) ---------------------------------------------- */
/* The reference has no derivative code: these entries have no counterpart in
 * it.  They differentiate its forward map, the SIB step of the dynamics
 * (dynamics/spindynamics.f90:282-313 stage loop) with the effective field of
 * Hamiltonian_type/hamiltonian_collection.f90:433-454, on single-atom stencil
 * plans without the dipolar term.  The differentiable coupling terms are the
 * J, D and K terms of the plan's mj_hamiltonian_desc in that order (nJ + nD + nK
 * values, at most 8); the field is linear in their values. */
mj_status mj_plan_nterms(const mj_plan* plan, int32_t* nterms);
/* Re-set the term values (the `value` fields, in the same order) of a stencil plan. */
mj_status mj_plan_set_terms(mj_plan* plan, const double* values);
/* VJP of get_eff_field at m (device SoA) for the cotangent v: g_m = (dB/dm)^T v,
 * g_terms[t] = v . dB/dvalue_t (device, nterms doubles), g_b = (dB/db)^T v per
 * site (device SoA, the applied-field map); each output may be NULL. */
mj_status mj_field_vjp(mj_plan* plan, const double* m_dev_soa, const double* v_dev_soa, double* g_m_dev_soa,
                       double* g_terms_dev, double* g_b_dev_soa, void* stream);
/* A reverse-mode trajectory of `nsteps` SIB steps, checkpointed every
 * `checkpoint_every` steps (each segment is recomputed in the backward sweep). */
typedef struct mj_adjoint mj_adjoint;
mj_status mj_adjoint_create(mj_plan* plan, int32_t nsteps, int32_t checkpoint_every, mj_adjoint** out);
mj_status mj_adjoint_destroy(mj_adjoint* a);
/* m_T from m_0 (device SoA; p: MJ_SIB, any noise mode), keeping the checkpoints. */
mj_status mj_adjoint_forward(mj_adjoint* a, const mj_dyn_params* p, const double* m0_dev_soa, double* mT_dev_soa,
                             void* stream);
/* Given dL/dm_T, the gradients of the last forward: dL/dm_0, dL/dvalue_t
 * (device, nterms doubles, may be NULL) and dL/db per site (device SoA, may be NULL). */
mj_status mj_adjoint_backward(mj_adjoint* a, const double* gT_dev_soa, double* g0_dev_soa, double* g_terms_dev,
                              double* g_b_dev_soa, void* stream);

/* ---- batched replicas ---------------------------------------------------- */
/* Many independent 2D replicas of one single-atom Hamiltonian (the cell, shells
 * and couplings of `cell`/`ham`), each with its own size L[2r], L[2r+1], applied
 * field B_ext[3r..3r+2] (T) and temperature[r] (K), advanced by SIB in one
 * persistent launch per stage.  In the reference every such replica is a
 * separate run of the dynamics (dynamics/spindynamics.f90:260-323), one per MPI
 * rank group for parallel tempering (paratemp-MC/parallel_tempering.f90:24-217).
 * Spins are packed SoA: x[Ntot] | y[Ntot] | z[Ntot], replica r at sites
 * [off_r, off_r+1) of mj_batch_nsites.  Replica r draws Philox noise on stream
 * p->stream_id + r with its local site index, so it reproduces a plan of its
 * own size run with stream_id + r.  The dipolar term is not batched. */
typedef struct mj_batch mj_batch;
mj_status mj_batch_create(const mj_lattice_desc* cell, const mj_hamiltonian_desc* ham, int32_t nrep,
                          const int32_t* L, const double* B_ext, const double* temperature,
                          int32_t device, mj_batch** out);
mj_status mj_batch_destroy(mj_batch* b);
/* Ntot and, if offsets != NULL, nrep+1 packed offsets. */
mj_status mj_batch_nsites(const mj_batch* b, int64_t* total, int64_t* offsets);
mj_status mj_batch_device_ptr(const mj_batch* b, double** m_dev_soa);
/* Host AoS (3, Ntot) in replica order (asynchronous upload, synchronous download). */
mj_status mj_batch_upload(mj_batch* b, const double* m_host_aos, void* stream);
mj_status mj_batch_download(const mj_batch* b, double* m_host_aos, void* stream);
/* nsteps SIB steps of every replica (p->integrator must be MJ_SIB, noise OFF or
 * PHILOX, p->temperature is ignored: each replica has its own).  With
 * swap_every > 0, after every step s with (s+1) % swap_every == 0 the replica
 * energies are evaluated and one parallel-tempering round runs on the ladder of
 * temperatures: paratemp-MC/paratemp.f90:47-103 (reorder_temperature: pairs
 * (l, l+1) from l = round % 2 in steps of 2) and :105-119 (accept: delta =
 * (1/kT_{l+1} - 1/kT_l)(E_{l+1} - E_l), accepted if > 0, else if
 * exp(max(delta,-200)) > u, u a Philox uniform); only neighbours of equal size
 * are compared; an accepted swap exchanges the two replicas' temperatures.
 * E_dev (device, nrep doubles, may be NULL) receives the energies after the
 * last step. */
mj_status mj_batch_step(mj_batch* b, const mj_dyn_params* p, int32_t nsteps, int32_t swap_every,
                        double* E_dev, void* stream);
/* The same as a CUDA graph of steps_per_graph steps (a multiple of swap_every,
 * p->step0 too) replayed nreplay times; steps advance p->step0 by
 * steps_per_graph per replay. */
mj_status mj_batch_graph_run(mj_batch* b, const mj_dyn_params* p, int32_t steps_per_graph, int32_t nreplay,
                             int32_t swap_every, double* E_dev, void* stream);
/* Energies (host, nrep) of the current state; synchronous. */
mj_status mj_batch_energies(mj_batch* b, double* E_host);
/* Current temperature of every replica (K) and, if accepted != NULL, the
 * accepted-swap count of every ladder pair (l, l+1) (reference Nsuccess). */
mj_status mj_batch_temperatures(const mj_batch* b, double* T_host, int32_t* accepted);
/* Field and energy of every replica at the batch's current state: get_eff_field
 * and H%energy per image as GNEB evaluates them (GNEB/gneb_utils.f90:77-81,
 * 154-157).  B_dev (device SoA, 3 Ntot, may be NULL) receives the effective
 * field, with the component along m removed when project != 0 (vec_project,
 * vector_utils/vector.f90:61-72); E_dev (device, nrep, may be NULL) the energies. */
mj_status mj_batch_field(mj_batch* b, double* B_dev_soa, double* E_dev, int32_t project, void* stream);
/* GNEB path tangents of replicas taken as the images of a path (all of one
 * size), into tau_dev (device SoA, 3 Ntot): mode 0 the energy-weighted tangent
 * of GNEB/tangent.f90:93-124 from the image energies E_dev (device, nrep), mode 1
 * the central difference of :163-180; end images take the one-sided
 * difference; each tangent is projected on the tangent space of its image and
 * normalised over the image. */
mj_status mj_batch_gneb_tangent(mj_batch* b, const double* E_dev, int32_t mode, double* tau_dev_soa, void* stream);
/* GNEB_input's path-relaxation part (IO-input/GNEB_io.f90): spring, vpo_dt,
 * vpo_mass, mep_ftol (or mep_ftol_ci), mep_itrmax, en_zero ('I', 'F' or 'N'),
 * climb != 0 for the climbing-image run (do_gneb_ci). */
typedef struct mj_gneb_params {
    double spring, dt, mass, ftol;
    int64_t itrmax;
    int32_t en_zero;
    int32_t climb;
} mj_gneb_params;

/* GNEB minimum-energy path of replicas taken as the images of a path (all of
 * one size, 3 or more; replica 0 and the last are the fixed end points): the
 * find_path relaxation of GNEB/gneb_utils.f90:19-240 on the batch's current
 * state, which it leaves holding the relaxed path.  Per iteration the interior
 * images move by velocity Verlet, r = m + v dt + F dt^2 / (2 mass) normalised;
 * F is the projected field minus its component along the energy-weighted
 * tangent plus the spring force spring (l_{i+1} + l_{i-1} - 2 l_i) along it,
 * l the geodesic path length; with climb, the first image of highest energy
 * (chosen again each iteration) takes F - 2 tau (F.tau) instead; velocity and
 * old force are carried along each spin's rotation, and the velocity is
 * projected on the force (VPO).  Stops when max |F| < ftol or after itrmax
 * iterations.  Host outputs (nrep each): rx the path length at every image,
 * ene the energy above image 0 (en_zero 'I'), the last image ('F') or zero
 * ('N'), dene the derivative of the energy along the path (en_path.out of
 * GNEB/io-gneb.f90:83-111); iterations, max_force and climbing (may be NULL)
 * the iterations taken, the final max |F| and the climbing image (0-based; -1
 * without climb).  Synchronous: starts after the work queued on the legacy
 * default stream, returns with the relaxed path in the batch. */
mj_status mj_batch_gneb_path(mj_batch* b, const mj_gneb_params* p, double* rx, double* ene, double* dene,
                             int64_t* iterations, double* max_force, int32_t* climbing);
/* The same relaxation (GNEB/gneb_utils.f90:19-240 find_path) on a path of
 * nimg images (3 or more) of any plan: the images' fields and energies are the
 * plan's own get_eff_field and H%energy (GNEB/gneb_utils.f90:77-81,154-157),
 * so every lattice and term a plan holds, the FFT dipolar term, 3D films and
 * ELL couplings included, reaches the GNEB.  One magnetic atom per cell, as
 * the reference requires (GNEB/gneb_utils.f90:69): MJ_ERR_UNSUPPORTED else.  m_dev (device,
 * nimg * 3 N doubles; image r the SoA block x[N] | y[N] | z[N] at 3 N r)
 * holds the path and receives the relaxed one.  Outputs as mj_batch_gneb_path.
 * Starts after the work queued on `stream` (the iterations run as CUDA graphs
 * on a stream of the plan's own) and returns with the path relaxed; at most
 * 65535 * 256 spins per image.  Replaces the GNEB driver's image loop over get_eff_field/energy
 * (GNEB/gneb_utils.f90:72-200) for a Hamiltonian held by a plan.  Returns
 * MJ_ERR_TIMEOUT when an image's field launch gave up a bounded wait during the
 * relaxation: the path and the outputs are then invalid. */
mj_status mj_gneb_path(mj_plan* plan, double* m_dev_images, int32_t nimg, const mj_gneb_params* p, double* rx,
                       double* ene, double* dene, int64_t* iterations, double* max_force, int32_t* climbing,
                       void* stream);
/* Tile variant (0: 32x16 tiles, 4 sites per thread; 1: 32x16, 2 per thread;
 * 2: 32x32, 4 per thread; 3: 32x8, 2 per thread, registers capped for 8
 * resident blocks of 4 warps; 4: 32x16, 2 per thread, capped for 4 blocks of 8
 * warps) and persistent blocks per SM (1..64). */
mj_status mj_batch_set_config(mj_batch* b, int32_t variant, int32_t blocks_per_sm);
/* Times `steps` steps of every (variant, blocks per SM in {2,4,8,16,32}) on the
 * current state (restored afterwards), keeps the fastest; ms_table (25 doubles,
 * may be NULL) gets ms per step in variant-major order. */
mj_status mj_batch_autotune(mj_batch* b, const mj_dyn_params* p, int32_t steps, int32_t* best_variant,
                            int32_t* best_blocks_per_sm, double* ms_table);
/* Parallel-tempering Monte Carlo on the replicas: the swap loop of
 * paratemp-MC/parallel_tempering.f90:163-181.  Each of nrounds rounds runs
 * sweeps_per_round Metropolis sweeps (mj_mc_sweeps' moves and colouring, one
 * colouring for every replica) of every replica at the temperature its ladder
 * slot holds, then measures (measure_add) and, when swap != 0, runs the
 * parallel-tempering round p->round0 + k of mj_batch_step's rule on those
 * energies.  Replica r is a chain of its own: Philox stream p->stream_id + r
 * with its local site index, its own cone and counts (first set from p->cone,
 * kept across calls; mj_batch_mc_reset sets them again).  p->temperature is
 * ignored, p->sweep0 and (with swaps) p->round0 advance.  Per round k:
 * E_dev[k nrep + r] the energy, M_dev[3 (k nrep + r) ..] the summed spins and
 * slot_dev[k nrep + r] the ladder slot of replica r during the round's sweeps
 * (each may be NULL); colors[4] as mj_mc_sweeps. */
mj_status mj_batch_mc(mj_batch* b, mj_mc_params* p, int32_t nrounds, int32_t sweeps_per_round, int32_t swap,
                      double* E_dev, double* M_dev, int32_t* slot_dev, int32_t* colors, void* stream);
/* Resets every replica's Monte Carlo chain state: cone, accepted and proposed counts. */
mj_status mj_batch_mc_reset(mj_batch* b, double cone);
/* Per-replica cone (rad), accepted and proposed moves (host arrays of nrep, each may be NULL). */
mj_status mj_batch_mc_state(mj_batch* b, double* cone, int64_t* accepted, int64_t* proposed);

#ifdef __cplusplus
}
#endif
#endif /* MATJES_GPU_H */
