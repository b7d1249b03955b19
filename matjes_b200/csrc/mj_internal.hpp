// Internal declarations shared by the host builder, the kernels and the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/matjes_gpu.h"

namespace mj {

// fixed-parameters/constant.f90:11-32
constexpr double kHbar = 0.658211928;         // eV fs
constexpr double kKB = 0.000086173324;        // eV / K
constexpr double kMuB = 0.0000578838180661;   // eV / T
constexpr double kDipPref = 6.745817653234234066975e-7;  // Energy/dipolar_magnetic.f90:41
constexpr double kPi = 3.14159265358979323846264338327950288;

constexpr int kMaxOff = 48;  // neighbour offsets held in the launch parameters

// One 3x3 coupling block of the "MM" Hamiltonian: rows = components of
// magnetic atom a in cell c, cols = components of magnetic atom b in cell c+o.
struct Block {
    int a, b;
    int o[3];
    double T[9];  // row-major
};

struct Geometry {
    mj_lattice_desc d;
    double pos[MJ_MAX_ATOMS][3];  // nm
    int magidx[MJ_MAX_ATOMS];
    int magatom[MJ_MAX_ATOMS];
    int nmag = 0;
};

// Host builder (mj_lattice.cpp).  Returns false with `err` set on failure.
bool build_geometry(const mj_lattice_desc& lat, Geometry& g, std::string& err);
bool build_blocks(const Geometry& g, const mj_hamiltonian_desc& ham, std::vector<Block>& blocks,
                  std::vector<double>& onsite /* 9*nmag*nmag, per (a,b) pair at o=0 */, std::string& err);
// Real-space dipolar K on the N_rep grid (Nmag = 1): K[k*9 + 3r + c].
bool build_dipolar_kernel(const Geometry& g, const mj_hamiltonian_desc& ham, int nrep[3],
                          std::vector<double>& K, std::string& err);

// Launch-parameter image of a single-atom stencil.  Passed by value
// (__grid_constant__) so that every plan can run without global state.
struct StencilParams {
    int L[3];
    int periodic[3];
    int n_off;
    int has_onsite;
    int off[kMaxOff][3];
    int iso[kMaxOff];         // 1 when W == w*I (pure exchange offset)
    double W[kMaxOff][9];     // B_i += W_o m_{i+o},  W_o = -(T_o + T_{-o}^T)
    double W0[9];             // on-site: -(T_0 + T_0^T)
    double zc;                // B_i += zc * b_cell,  zc = -(mu0 muB c_zeeman mu_s)
    double bext[3];
    int zee_on;
    int shape;                // mj_shapes.hpp ShapeId; W is then in the shape's offset order
};

// Dipolar H on the padded FFT grid (the unpack is fused into the consumers):
// component c of site (x,y,z) is h[c*cs + x + px*y + zs*z].
struct DipView {
    const double* h;
    int64_t cs;   // component stride
    int64_t zs;   // z-plane stride
    int px;       // padded x extent (row stride)
};

// The dipolar term's padded input grid (the layout of DipView): a step kernel
// given one stores every spin it writes there too, so that the next dipolar
// evaluation of those spins needs no pad launch.  p = null: none.
struct DipPad {
    double* p;
    int64_t cs;
    int64_t zs;
    int px;
};

// Dynamics coefficients computed once per call on the host.
struct DynCoef {
    int integrator;
    int thermal;
    int noise;
    double h_over_hbar;   // stage dt / hbar (Euler, Heun)
    double inv_den;       // 1/(1+alpha^2)
    double alpha;
    double sib_hc;        // -0.5 (dt/hbar)/(1+alpha^2)
    double sigma;         // sqrt(alpha kT hbar / dt_noise)
    uint64_t seed;
    uint32_t stream_id;
    const double* inject;
    int inject_nbuf;
    // graph replay: the thermal step index is *step_base + step (null = step)
    const uint32_t* step_base;
    uint32_t keys[20];          // Philox round keys of `seed`
    const double* noise_tab;    // device tables of the Box-Muller evaluation (kNoiseTabDoubles)
};

// Box-Muller tables (host-built, identical to the oracle's): 1024 (sin, cos) pairs
// of 2 pi (i + 1/2)/1024 followed by 1024 (1/F, ln F) pairs of F = 1 + (j + 1/2)/1024.
constexpr int kNoiseTabDoubles = 4096;
void build_noise_tables(double* tab);

}  // namespace mj

struct mj_plan {
    int device = 0;
    int64_t N = 0;        // spin sites
    int64_t ncell = 0;
    int nmag = 1;
    bool is_stencil = true;
    mj::StencilParams sp{};
    int tile_variant = 0;            // tiled-kernel shape (threads in y x sites per thread), see mj_tiled.cu
    int tiled_shape = 0;             // matched compile-time shape (sp.shape is 0 while the generic path is forced)
    bool use_tma = true;             // tiled kernels stage tile + halo with one TMA copy per block
    bool fused_sib = false;          // SIB steps of tiled plans without the dipolar term in one launch
    bool use_pdl = true;             // tiled passes launched as programmatic dependents of the kernel before
    bool store_draw = true;          // SIB: the predictor stores its Philox draw for the corrector (else recomputed)
    unsigned int* d_sched = nullptr; // fused step scheduler: work counter, exit ticket, done tiles per row
    int num_sms = 148;
    int* d_status = nullptr;         // device status word: kStatusTimeout | kStatusNonFinite
    int* h_status = nullptr;         // pinned host copy of it (host-array step calls)
    int defer_nblocks = 0;           // energy partials written by the last pass launched with emode 1
    // ELL form (multi-atom cells, COO input): width entries per site
    int ell_width = 0;
    int* d_ell_col = nullptr;        // [width][N], -1 = empty
    double* d_ell_val = nullptr;     // [width][9][N]
    double* d_zee = nullptr;         // per-site Zeeman coefficient zc (ELL)
    // applied field map (SoA per cell) or null for uniform
    double* d_bmap = nullptr;
    std::vector<double> bext_cell;   // ELL uniform field
    // dipolar
    bool dip_on = false;
    int nrep[3] = {0, 0, 0};
    void* dip = nullptr;             // DipolarPlan (mj_dipolar.cu)
    // scratch
    double* d_mid = nullptr;         // 3N
    double* d_aux = nullptr;         // 3N (Heun D1)
    double* d_aux2 = nullptr;        // 3N (Heun DT)
    double* d_field = nullptr;       // 3N (field scratch)
    double* d_partials = nullptr;    // per-block energy partials
    unsigned int* d_counter = nullptr;
    double* d_scalar = nullptr;      // 8 doubles of device scratch
    double* d_noise_tab = nullptr;   // Box-Muller tables (kNoiseTabDoubles)
    int64_t partial_cap = 0;
    // host-array convenience calls (allocated on first use)
    double* d_stage = nullptr;       // 3N AoS staging
    double* d_tmp_m = nullptr;       // 3N
    double* d_tmp_b = nullptr;       // 3N
    double* d_tmp_e = nullptr;       // N + 8
    // CUDA graph of a step loop (mj_graph_run), cached with the key it was captured for
    uint32_t* d_stepctr = nullptr;
    cudaStream_t cap_stream = nullptr;
    // streams and events of the striped host-to-host step (mj_step_host)
    cudaStream_t pipe_stream[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // copies in, out, 4 compute
    std::vector<cudaEvent_t> pipe_events;
    cudaGraphExec_t graph_exec = nullptr;
    std::string graph_key;
    // the striped host-array step captured as a graph (mj_step_host), with its key
    cudaGraphExec_t host_graph_exec = nullptr;
    std::string host_graph_key;
    int host_stripes = 0;  // stripes of mj_step_host (0: the default)
    int blocks_per_sm = 0;    // cap on resident tiled-pass blocks per SM (0: none)
    bool dip_zconv = true;    // FFT dipolar: the fused z convolution where the grid allows it
    bool host_zerocopy = true;  // striped mj_step_host: downloads written by kernels into the mapped host buffer
    // FFT dipolar inside a step sequence: the step kernels also write their spins
    // into the padded grid, which then holds dip_pad_holds (null: unknown)
    bool dip_fuse_pad = false;
    const double* dip_pad_holds = nullptr;
    int smem_cap_bytes = 0;   // the dynamic shared memory per block that makes the cap
    // per-kernel event timing (mj_profile_enable / mj_profile_read)
    bool prof_on = false;
    struct ProfRec {
        int id;
        cudaEvent_t a, b;
    };
    std::vector<ProfRec> prof;
    std::vector<std::string> prof_names;
    std::vector<mj::Block> blocks;   // kept for the adjoint / introspection
    // differentiable coupling terms (stencil plans): the description the plan was
    // built from, and per-term unit stencils W_t (W = sum_t value_t W_t), built on
    // first use: [nterm][n_off + 1][9], on-site tensor last, offsets in sp order
    mj::Geometry geom;
    mj_hamiltonian_desc ham{};       // term pointers cleared; the terms are copied below
    std::vector<mj_exchange_term> termJ;
    std::vector<mj_dmi_term> termD;
    std::vector<mj_aniso_term> termK;
    std::vector<double> unitW;
    double* d_unit = nullptr;
    double* d_vjp_part = nullptr;          // term-gradient reduction scratch of mj_field_vjp
    unsigned int* d_vjp_counter = nullptr;
};

struct mj_state {
    const mj_plan* plan = nullptr;
    double* d_m = nullptr;  // SoA 3N
};

namespace mj {
// Bits of a plan's device status word (read and cleared by mj_plan_check_status):
// a bounded device wait gave up; a step wrote a non-finite spin component.
constexpr int kStatusTimeout = 1;
constexpr int kStatusNonFinite = 2;
// The error a status word reports (MJ_OK for 0); a non-zero word is cleared on
// the device and the energy ticket counter re-armed (mj_abi.cpp).
mj_status status_from_word(mj_plan* p, int word);

// error reporting (mj_abi.cpp)
mj_status set_error(mj_status st, const std::string& msg);
mj_status cuda_status(cudaError_t e, const char* where);

// per-kernel timing records (mj_abi.cpp); prof_begin returns -1 when not recording
int prof_begin(mj_plan* p, const char* name, cudaStream_t s);
void prof_end(mj_plan* p, int rec, cudaStream_t s);

// kernel launchers (mj_kernels.cu)
mj_status launch_field(mj_plan* p, const double* m, double* B, double* e_site, double* E_out, cudaStream_t s);
// one time step; Euler writes m_out, the two-pass schemes update m in place
mj_status launch_step(mj_plan* p, double* m, double* m_out, const DynCoef& c, uint32_t step, double* E_prev_out,
                      cudaStream_t s);
mj_status launch_energy(mj_plan* p, const double* m, double* E_out, cudaStream_t s);
mj_status launch_philox(uint64_t seed, uint32_t step, uint32_t stream_id, int64_t n, double* out, cudaStream_t s);
mj_status launch_temperature(mj_plan* p, const double* m, double* out2 /* device: [sum|mxB|^2, sum m.B] */, cudaStream_t s);
mj_status step_counter(uint32_t* ctr, uint32_t value, bool add, cudaStream_t s);
mj_status aos_to_soa(const double* src_aos, double* dst_soa, int64_t n, cudaStream_t s);
mj_status soa_to_aos(const double* src_soa, double* dst_aos, int64_t n, cudaStream_t s);
// the transposes restricted to the sites [i0, i0 + cnt) of n
mj_status aos_to_soa_range(const double* src_aos, double* dst_soa, int64_t i0, int64_t cnt, int64_t n, cudaStream_t s);
mj_status soa_to_aos_range(const double* src_soa, double* dst_aos, int64_t i0, int64_t cnt, int64_t n, cudaStream_t s);
// the same into a mapped host buffer (sites staged per block, contiguous writes)
mj_status soa_to_aos_stream(const double* src_soa, double* dst_aos, int64_t i0, int64_t cnt, int64_t n, cudaStream_t s);
// one block of nthreads sums nblocks energy partials in ordered_sum's fixed order
mj_status launch_ordered_sum(const double* partials, int nblocks, int nthreads, double* out, cudaStream_t s);
int64_t energy_blocks(const mj_plan* p);

// tiled kernels for compile-time stencil shapes (mj_tiled.cu dispatches to one
// translation unit per shape, mj_tiled_<shape>.cu)
// pass: 0 field, 1 euler, 2 heun1, 3 heun2, 4 sib1, 5 sib2
constexpr int kTiledVariants = 6;
constexpr int kTiledVariantTY[kTiledVariants] = {16, 32, 16, 16, 16, 8};  // tile height per variant
constexpr int kTiledVariantBYT[kTiledVariants] = {4, 8, 8, 4, 8, 4};     // warps per block per variant
// emode: energy reduction of the launch (0: into E_out at once; 1: per-block
// partials only, counted in p->defer_nblocks; 2: block 0 sums the previous
// pass's partials into E_out).  nty >= 0 limits the launch to the tile rows
// [ty0, ty0 + nty) (plain staging; block ids and energy partials those of the
// whole-lattice launch, so emode 1 over all row ranges writes the same partials).
mj_status launch_tiled(mj_plan* p, int pass, const DynCoef& C, const double* ms, const double* mn, double* out,
                       double* aux, double* aux2, DipView Hd, double* E_out, uint32_t step, cudaStream_t s,
                       int emode = 0, int ty0 = 0, int nty = -1);
#define MJ_TILED_SHAPE_DECL(fn)                                                                                   \
    mj_status fn(mj_plan* p, int pass, const DynCoef& C, const double* ms, const double* mn, double* out,         \
                 double* aux, double* aux2, DipView Hd, double* E_out, uint32_t step, cudaStream_t s, int emode,  \
                 int ty0, int nty);
// one SIB step in one launch (k_sib_fused): tiled plans without the dipolar term
mj_status launch_sib_fused(mj_plan* p, const DynCoef& C, double* m, double* draw, double* E_out, uint32_t step,
                           cudaStream_t s);
#define MJ_FUSED_SHAPE_DECL(fn) \
    mj_status fn(mj_plan* p, const DynCoef& C, double* m, double* draw, double* E_out, uint32_t step, cudaStream_t s);
MJ_FUSED_SHAPE_DECL(launch_sib_fused_square_nn)
MJ_FUSED_SHAPE_DECL(launch_sib_fused_square2)
MJ_FUSED_SHAPE_DECL(launch_sib_fused_tri_nn)
MJ_FUSED_SHAPE_DECL(launch_sib_fused_tri3)
// The GNEB images of a path on a tiled plan without the dipolar term: the
// projected field into F and per tile the six path sums and the energy
// (partials[q nblocks + tile], tiles image-major, *tiles_per_image of them).
mj_status launch_gneb_images(mj_plan* p, const double* m, double* F, double* partials, int nimg,
                             int64_t* tiles_per_image, cudaStream_t s);
#define MJ_GNEB_SHAPE_DECL(name)                                                                       \
    mj_status name(mj_plan* p, const double* m, double* F, double* partials, int nimg, int64_t* tiles, \
                   cudaStream_t s);
MJ_GNEB_SHAPE_DECL(launch_gneb_images_square_nn)
MJ_GNEB_SHAPE_DECL(launch_gneb_images_square2)
MJ_GNEB_SHAPE_DECL(launch_gneb_images_tri_nn)
MJ_GNEB_SHAPE_DECL(launch_gneb_images_tri3)
// scheduler words of the fused step: 2 + tile rows at the smallest tile height
int64_t sched_words(const mj_plan* p);
MJ_TILED_SHAPE_DECL(launch_tiled_square_nn)
MJ_TILED_SHAPE_DECL(launch_tiled_square2)
MJ_TILED_SHAPE_DECL(launch_tiled_tri_nn)
MJ_TILED_SHAPE_DECL(launch_tiled_tri3)
int64_t tiled_energy_blocks(const mj_plan* p);
// tile rows of the tiled kernels (per variant height) over the lattice
int tiled_tile_rows(const mj_plan* p);
// match a single-atom stencil to a compile-time shape and reorder its tensors (mj_abi.cpp)
void match_shape(mj::StencilParams& sp);
// single-atom stencil tensors W_o from coupling blocks; false past kMaxOff offsets (mj_abi.cpp)
bool stencil_from_blocks(const std::vector<Block>& blocks, const std::vector<double>& onsite, StencilParams& sp);
// dynamics coefficients of a plan, validated (mj_abi.cpp)
mj_status make_dyn_coef(const mj_dyn_params* d, const mj_plan* plan, DynCoef& c);
// drop a plan's captured step graph (after its launch parameters change)
void drop_graph(mj_plan* p);

// dipolar (mj_dipolar.cu)
mj_status dipolar_create(mj_plan* p, const std::vector<double>& K, cudaStream_t s);
void dipolar_destroy(mj_plan* p);
// H = K * m on the padded grid; consumers read it through dipolar_view and fold B -= 2H.
mj_status dipolar_apply(mj_plan* p, const double* m, double* H_unused, cudaStream_t s);
DipPad dipolar_pad(const mj_plan* p);
DipView dipolar_view(const mj_plan* p);
}  // namespace mj
