// C ABI of the B200 Matjes hot path: plans, states, field, energy, steps.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "mj_internal.hpp"
#include "mj_shapes.hpp"

namespace mj {

static thread_local std::string g_err = "no error";

mj_status set_error(mj_status st, const std::string& msg) {
    g_err = msg;
    return st;
}

mj_status cuda_status(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return MJ_OK;
    const mj_status st = (e == cudaErrorMemoryAllocation) ? MJ_ERR_OOM : MJ_ERR_CUDA;
    return set_error(st, std::string(where) + ": " + cudaGetErrorString(e));
}

void match_shape(StencilParams& sp);

mj_status status_from_word(mj_plan* p, int word) {
    if (word == 0) return MJ_OK;
    // clear the word; re-arm the ticket counter of the energy reduction, which a
    // launch that failed may have left part-way
    cudaMemset(p->d_status, 0, sizeof(int));
    cudaMemset(p->d_counter, 0, 4 * sizeof(unsigned int));
    if (word & kStatusTimeout)
        return set_error(MJ_ERR_TIMEOUT, "a bounded device wait (TMA mbarrier) gave up; results of that launch are invalid");
    return set_error(MJ_ERR_NAN, "a time step wrote a non-finite spin component; the state is invalid from that step on");
}

int prof_begin(mj_plan* p, const char* name, cudaStream_t s) {
    if (!p->prof_on) return -1;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return -1;
    int id = -1;
    for (size_t k = 0; k < p->prof_names.size(); ++k)
        if (p->prof_names[k] == name) id = static_cast<int>(k);
    if (id < 0) {
        id = static_cast<int>(p->prof_names.size());
        p->prof_names.push_back(name);
    }
    mj_plan::ProfRec r;
    r.id = id;
    if (cudaEventCreate(&r.a) != cudaSuccess) return -1;
    if (cudaEventCreate(&r.b) != cudaSuccess) {
        cudaEventDestroy(r.a);
        return -1;
    }
    cudaEventRecord(r.a, s);
    p->prof.push_back(r);
    return static_cast<int>(p->prof.size() - 1);
}

void prof_end(mj_plan* p, int rec, cudaStream_t s) {
    if (rec < 0 || rec >= static_cast<int>(p->prof.size())) return;
    cudaEventRecord(p->prof[rec].b, s);
}

namespace {

void prof_clear(mj_plan* p) {
    for (auto& r : p->prof) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    p->prof.clear();
    p->prof_names.clear();
}

template <class T>
mj_status dalloc(T** p, size_t n, const char* what) {
    *p = nullptr;
    if (n == 0) return MJ_OK;
    return cuda_status(cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)), what);
}

void transpose3(const double* T, double* Tt) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Tt[3 * c + r] = T[3 * r + c];
}

bool same_off(const int* a, const int* b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; }

// Single-atom stencil: W_o = -(T_o + T_{-o}^T) for every offset of the shell set.
bool make_stencil(const std::vector<Block>& blocks, const std::vector<double>& onsite, StencilParams& sp) {
    std::vector<std::array<int, 3>> offs;
    auto find_T = [&](const int* o, double* T) {
        std::fill(T, T + 9, 0.0);
        bool f = false;
        for (const Block& b : blocks)
            if (same_off(b.o, o)) {
                for (int k = 0; k < 9; ++k) T[k] = T[k] + b.T[k];
                f = true;
            }
        return f;
    };
    double T0[9];
    for (int k = 0; k < 9; ++k) T0[k] = onsite[k];
    for (const Block& b : blocks) {
        if (b.o[0] == 0 && b.o[1] == 0 && b.o[2] == 0) {
            for (int k = 0; k < 9; ++k) T0[k] += b.T[k];
            continue;
        }
        std::array<int, 3> o = {b.o[0], b.o[1], b.o[2]};
        std::array<int, 3> mo = {-b.o[0], -b.o[1], -b.o[2]};
        if (std::find(offs.begin(), offs.end(), o) == offs.end()) offs.push_back(o);
        if (std::find(offs.begin(), offs.end(), mo) == offs.end()) offs.push_back(mo);
    }
    if (static_cast<int>(offs.size()) > kMaxOff) return false;
    sp.n_off = static_cast<int>(offs.size());
    for (int k = 0; k < sp.n_off; ++k) {
        const int o[3] = {offs[k][0], offs[k][1], offs[k][2]};
        const int mo[3] = {-o[0], -o[1], -o[2]};
        double T[9], Tm[9], Tmt[9];
        find_T(o, T);
        find_T(mo, Tm);
        transpose3(Tm, Tmt);
        bool iso = true;
        for (int q = 0; q < 9; ++q) {
            sp.W[k][q] = -(T[q] + Tmt[q]);
            const bool diag = (q == 0 || q == 4 || q == 8);
            if (!diag && sp.W[k][q] != 0.0) iso = false;
        }
        if (!(sp.W[k][0] == sp.W[k][4] && sp.W[k][0] == sp.W[k][8])) iso = false;
        sp.iso[k] = iso ? 1 : 0;
        for (int d = 0; d < 3; ++d) sp.off[k][d] = o[d];
    }
    double T0t[9];
    transpose3(T0, T0t);
    sp.has_onsite = 0;
    for (int q = 0; q < 9; ++q) {
        sp.W0[q] = -(T0[q] + T0t[q]);
        if (sp.W0[q] != 0.0) sp.has_onsite = 1;
    }
    return true;
}

// Reorder a stencil into the offset order of a compile-time shape, if its
// offset set is the shape's (in-plane only) and every offset the shape treats
// as isotropic is isotropic here.
template <class S>
bool try_shape(StencilParams& sp) {
    if (sp.n_off != S::K) return false;
    int perm[kMaxOff];
    for (int k = 0; k < S::K; ++k) {
        int j = -1;
        for (int q = 0; q < sp.n_off; ++q)
            if (sp.off[q][0] == S::DX[k] && sp.off[q][1] == S::DY[k] && sp.off[q][2] == 0) j = q;
        if (j < 0 || (S::ISO[k] && !sp.iso[j])) return false;
        perm[k] = j;
    }
    StencilParams o = sp;
    for (int k = 0; k < S::K; ++k) {
        for (int d = 0; d < 3; ++d) sp.off[k][d] = o.off[perm[k]][d];
        for (int q = 0; q < 9; ++q) sp.W[k][q] = o.W[perm[k]][q];
        sp.iso[k] = o.iso[perm[k]];
    }
    sp.shape = S::id;
    return true;
}

struct Entry {
    int64_t row, col;
    double W[9];
};

// Per-site tensor lists (ELL) from (row site, col site, H block) triplets:
// B_s = -sum_t (H_st + H_ts^T) m_t.
mj_status make_ell(mj_plan* p, std::vector<Entry>& ent) {
    std::sort(ent.begin(), ent.end(), [](const Entry& a, const Entry& b) {
        return a.row != b.row ? a.row < b.row : a.col < b.col;
    });
    std::vector<Entry> merged;
    for (const Entry& e : ent) {
        if (!merged.empty() && merged.back().row == e.row && merged.back().col == e.col) {
            for (int q = 0; q < 9; ++q) merged.back().W[q] += e.W[q];
        } else {
            merged.push_back(e);
        }
    }
    const int64_t N = p->N;
    std::vector<int> count(N, 0);
    for (const Entry& e : merged) ++count[e.row];
    int width = 0;
    for (int c : count) width = std::max(width, c);
    p->ell_width = width;
    std::vector<int> col(static_cast<size_t>(width) * N, -1);
    std::vector<double> val(static_cast<size_t>(width) * 9 * N, 0.0);
    std::vector<int> fill(N, 0);
    for (const Entry& e : merged) {
        const int k = fill[e.row]++;
        col[static_cast<size_t>(k) * N + e.row] = static_cast<int>(e.col);
        for (int q = 0; q < 9; ++q) val[(static_cast<size_t>(k) * 9 + q) * N + e.row] = e.W[q];
    }
    mj_status st;
    if ((st = dalloc(&p->d_ell_col, col.size(), "ell col")) != MJ_OK) return st;
    if ((st = dalloc(&p->d_ell_val, val.size(), "ell val")) != MJ_OK) return st;
    if (!col.empty()) {
        if ((st = cuda_status(cudaMemcpy(p->d_ell_col, col.data(), col.size() * sizeof(int), cudaMemcpyHostToDevice),
                              "ell col upload")) != MJ_OK)
            return st;
        if ((st = cuda_status(cudaMemcpy(p->d_ell_val, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice),
                              "ell val upload")) != MJ_OK)
            return st;
    }
    return MJ_OK;
}

void push_pair(std::vector<Entry>& ent, int64_t s, int64_t t, const double* H) {
    Entry f;
    f.row = s;
    f.col = t;
    for (int q = 0; q < 9; ++q) f.W[q] = -H[q];
    ent.push_back(f);
    Entry r;
    r.row = t;
    r.col = s;
    double Ht[9];
    transpose3(H, Ht);
    for (int q = 0; q < 9; ++q) r.W[q] = -Ht[q];
    ent.push_back(r);
}

mj_status ell_from_blocks(mj_plan* p, const Geometry& g, const std::vector<Block>& blocks, const std::vector<double>& onsite) {
    const int nm = g.nmag;
    const int* L = g.d.L;
    std::vector<Entry> ent;
    for (int64_t c = 0; c < p->ncell; ++c) {
        const int x = static_cast<int>(c % L[0]);
        const int y = static_cast<int>((c / L[0]) % L[1]);
        const int z = static_cast<int>(c / (static_cast<int64_t>(L[0]) * L[1]));
        for (const Block& b : blocks) {
            int n[3] = {x + b.o[0], y + b.o[1], z + b.o[2]};
            bool ok = true;
            for (int d = 0; d < 3; ++d) {
                if (n[d] < 0 || n[d] >= L[d]) {
                    if (!g.d.periodic[d]) ok = false;
                    n[d] = ((n[d] % L[d]) + L[d]) % L[d];
                }
            }
            if (!ok) continue;
            const int64_t c2 = n[0] + static_cast<int64_t>(L[0]) * (n[1] + static_cast<int64_t>(L[1]) * n[2]);
            push_pair(ent, c * nm + b.a, c2 * nm + b.b, b.T);
        }
        for (int a = 0; a < nm; ++a)
            for (int b = 0; b < nm; ++b) {
                const double* T = &onsite[(static_cast<size_t>(a) * nm + b) * 9];
                bool nz = false;
                for (int q = 0; q < 9; ++q) nz = nz || T[q] != 0.0;
                if (nz) push_pair(ent, c * nm + a, c * nm + b, T);
            }
    }
    return make_ell(p, ent);
}

mj_status alloc_scratch(mj_plan* p) {
    const int64_t N = p->N;
    mj_status st;
    if ((st = dalloc(&p->d_mid, 3 * N, "mid")) != MJ_OK) return st;
    if ((st = dalloc(&p->d_aux, 3 * N, "aux")) != MJ_OK) return st;
    if ((st = dalloc(&p->d_aux2, 3 * N, "aux2")) != MJ_OK) return st;
    // generic grid, or the smallest tile of the tiled kernels (32 x 8), whichever has more blocks
    const int64_t tiled_max = p->is_stencil ? static_cast<int64_t>((p->sp.L[0] + 31) / 32) * ((p->sp.L[1] + 7) / 8) * p->sp.L[2] : 0;
    p->partial_cap = 2 * std::max(energy_blocks(p), tiled_max) + 64;
    if ((st = dalloc(&p->d_partials, static_cast<size_t>(p->partial_cap), "partials")) != MJ_OK) return st;
    if ((st = dalloc(&p->d_counter, 4, "counter")) != MJ_OK) return st;
    if ((st = cuda_status(cudaMemset(p->d_counter, 0, 4 * sizeof(unsigned int)), "counter init")) != MJ_OK) return st;
    if (p->is_stencil) {
        const int64_t words = sched_words(p);
        if ((st = dalloc(&p->d_sched, words, "fused-step scheduler")) != MJ_OK) return st;
        if ((st = cuda_status(cudaMemset(p->d_sched, 0, sizeof(unsigned int) * words), "scheduler init")) != MJ_OK)
            return st;
    }
    if ((st = dalloc(&p->d_scalar, 8, "scalar")) != MJ_OK) return st;
    if ((st = dalloc(&p->d_status, 4, "status")) != MJ_OK) return st;
    if ((st = cuda_status(cudaMemset(p->d_status, 0, 4 * sizeof(int)), "status init")) != MJ_OK) return st;
    cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device);
    std::vector<double> tab(kNoiseTabDoubles);
    build_noise_tables(tab.data());
    if ((st = dalloc(&p->d_noise_tab, kNoiseTabDoubles, "noise tables")) != MJ_OK) return st;
    return cuda_status(cudaMemcpy(p->d_noise_tab, tab.data(), sizeof(double) * kNoiseTabDoubles, cudaMemcpyHostToDevice),
                       "noise tables");
}

void free_plan(mj_plan* p) {
    if (!p) return;
    if (p->dip) dipolar_destroy(p);
    prof_clear(p);
    if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
    if (p->host_graph_exec) cudaGraphExecDestroy(p->host_graph_exec);
    if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
    for (cudaStream_t& ps : p->pipe_stream)
        if (ps) cudaStreamDestroy(ps);
    for (cudaEvent_t e : p->pipe_events) cudaEventDestroy(e);
    cudaFree(p->d_stepctr);
    cudaFree(p->d_ell_col);
    cudaFree(p->d_ell_val);
    cudaFree(p->d_zee);
    cudaFree(p->d_bmap);
    cudaFree(p->d_mid);
    cudaFree(p->d_aux);
    cudaFree(p->d_aux2);
    cudaFree(p->d_field);
    cudaFree(p->d_partials);
    cudaFree(p->d_counter);
    cudaFree(p->d_scalar);
    cudaFree(p->d_status);
    cudaFree(p->d_sched);
    if (p->h_status) cudaFreeHost(p->h_status);
    cudaFree(p->d_noise_tab);
    cudaFree(p->d_stage);
    cudaFree(p->d_tmp_m);
    cudaFree(p->d_tmp_b);
    cudaFree(p->d_tmp_e);
    cudaFree(p->d_unit);
    cudaFree(p->d_vjp_part);
    cudaFree(p->d_vjp_counter);
    delete p;
}

mj_status ensure_host_scratch(mj_plan* p) {
    mj_status st;
    const int64_t N = p->N;
    if (!p->d_stage && (st = dalloc(&p->d_stage, 3 * N, "stage")) != MJ_OK) return st;
    if (!p->d_tmp_m && (st = dalloc(&p->d_tmp_m, 3 * N, "tmp m")) != MJ_OK) return st;
    if (!p->d_tmp_b && (st = dalloc(&p->d_tmp_b, 3 * N, "tmp b")) != MJ_OK) return st;
    if (!p->d_tmp_e && (st = dalloc(&p->d_tmp_e, N + 8, "tmp e")) != MJ_OK) return st;
    if (!p->h_status) {
        if ((st = cuda_status(cudaHostAlloc(&p->h_status, 32, cudaHostAllocDefault), "status mirror")) != MJ_OK)
            return st;
        std::memset(p->h_status, 0, 32);
    }
    return MJ_OK;
}

mj_status dyn_coef(const mj_dyn_params* d, const mj_plan* plan, DynCoef& c) {
    if (!d) return set_error(MJ_ERR_ARG, "null dynamics parameters");
    std::memset(&c, 0, sizeof(c));  // padding too: graphs are keyed by these bytes
    if (d->integrator != MJ_EULER && d->integrator != MJ_HEUN_MATJES && d->integrator != MJ_SIB)
        return set_error(MJ_ERR_ARG, "integrator must be MJ_EULER, MJ_HEUN_MATJES or MJ_SIB");
    if (!(d->timestep > 0.0) || !std::isfinite(d->timestep)) return set_error(MJ_ERR_ARG, "timestep must be > 0");
    if (!(d->alpha >= 0.0) || !(d->temperature >= 0.0)) return set_error(MJ_ERR_ARG, "alpha and temperature must be >= 0");
    if (d->noise < MJ_NOISE_OFF || d->noise > MJ_NOISE_INJECT) return set_error(MJ_ERR_ARG, "unknown noise mode");
    const int nloop = d->integrator == MJ_HEUN_MATJES ? 2 : 1;
    const double dt = d->timestep / static_cast<double>(nloop);  // dynamics/spindynamics.f90:266
    const double kT = d->temperature * kKB;
    c.integrator = d->integrator;
    c.noise = d->noise;
    c.thermal = (kT * d->alpha > 1e-10) && (kT > 1e-8) && d->noise != MJ_NOISE_OFF;
    c.alpha = d->alpha;
    c.inv_den = 1.0 / (1.0 + d->alpha * d->alpha);
    c.h_over_hbar = dt / kHbar;
    c.sib_hc = -0.5 * (d->timestep / kHbar) / (1.0 + d->alpha * d->alpha);
    c.sigma = std::sqrt(d->alpha * kT * kHbar / dt);
    c.seed = d->seed;
    c.stream_id = d->stream_id;
    c.inject = d->inject;
    c.inject_nbuf = d->inject_nbuf;
    c.step_base = nullptr;
    uint32_t k0 = static_cast<uint32_t>(d->seed), k1 = static_cast<uint32_t>(d->seed >> 32);
    for (int r = 0; r < 10; ++r) {  // Philox4x32 key schedule (Weyl increments)
        c.keys[2 * r] = k0;
        c.keys[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    c.noise_tab = plan->d_noise_tab;
    if (c.thermal && d->noise == MJ_NOISE_INJECT && (!d->inject || d->inject_nbuf < 1))
        return set_error(MJ_ERR_ARG, "MJ_NOISE_INJECT needs a device buffer and inject_nbuf >= 1");
    return MJ_OK;
}

// The step sequence shared by mj_step and the graph capture of mj_graph_run.
// Energies: MJ_ENERGY_AFTER gives E after step k in E_dev[k] (the energy of
// step k+1's incoming state, fused into its first pass, plus one extra field
// pass for the last step); MJ_ENERGY_BEFORE gives the incoming energies only.
// Euler alternates between m and the plan's midpoint buffer.
mj_status step_sequence(mj_plan* p, double* m, const DynCoef& c, int energy_mode, uint32_t step0, int32_t nsteps,
                        double* E_dev, cudaStream_t s) {
    mj_status st = MJ_OK;
    double* cur = m;
    double* other = p->d_mid;
    // the step kernels keep the dipolar pad grid current for the next
    // evaluation only within this sequence (the caller may change m between calls)
    struct PadScope {
        mj_plan* p;
        explicit PadScope(mj_plan* q) : p(q) {
            p->dip_fuse_pad = true;
            p->dip_pad_holds = nullptr;
        }
        ~PadScope() {
            p->dip_fuse_pad = false;
            p->dip_pad_holds = nullptr;
        }
    } pad_scope(p);
    for (int32_t k = 0; k < nsteps; ++k) {
        double* E = nullptr;
        if (E_dev) {
            if (energy_mode == MJ_ENERGY_BEFORE) E = E_dev + k;
            else if (k > 0) E = E_dev + (k - 1);
        }
        if ((st = launch_step(p, cur, other, c, step0 + static_cast<uint32_t>(k), E, s)) != MJ_OK) return st;
        if (c.integrator == MJ_EULER) std::swap(cur, other);
    }
    if (cur != m &&
        (st = cuda_status(cudaMemcpyAsync(m, cur, sizeof(double) * 3 * p->N, cudaMemcpyDeviceToDevice, s), "euler copy")) != MJ_OK)
        return st;
    if (E_dev && nsteps > 0 && energy_mode != MJ_ENERGY_BEFORE) return launch_energy(p, m, E_dev + (nsteps - 1), s);
    return MJ_OK;
}

}  // namespace

bool stencil_from_blocks(const std::vector<Block>& blocks, const std::vector<double>& onsite, StencilParams& sp) {
    return make_stencil(blocks, onsite, sp);
}

mj_status make_dyn_coef(const mj_dyn_params* d, const mj_plan* plan, DynCoef& c) { return dyn_coef(d, plan, c); }

void drop_graph(mj_plan* p) {
    if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
    p->graph_exec = nullptr;
    p->graph_key.clear();
    if (p->host_graph_exec) cudaGraphExecDestroy(p->host_graph_exec);
    p->host_graph_exec = nullptr;
    p->host_graph_key.clear();
}

void match_shape(StencilParams& sp) {
    sp.shape = kShapeGeneric;
    if (try_shape<ShapeTri3>(sp)) return;
    if (try_shape<ShapeTriNN>(sp)) return;
    if (try_shape<ShapeSquareNN>(sp)) return;
    try_shape<ShapeSquare2>(sp);
}

namespace {

// One step of host spins to host spins with the copies, the transposes and the
// passes cut into K stripes of tile rows, so that the upload of late stripes
// runs while early ones compute and download (the host link is full duplex).
// The passes of a step form a chain: each reads the previous one's output
// through the stencil, which reaches ry <= TY rows, so at most one tile row
// away.  Pass q of Q therefore runs over its stripe's tile rows shifted up by
// Q - 1 - q: stripe k's passes then need only the output of stripes <= k, and
// its first pass only the rows below 8 (t_{k+1} + Q - 1) + ry, which is what
// upload chunk k holds.  Every stripe waits for its own upload alone, one
// compute stream runs the stripes in order, and the copies stay few and large:
// a copy engine overlaps opposite copies of >= 6 MB almost fully, of 2 MB only
// in part (measured on a B200 over PCIe: 0.54 ms for 4 + 4 chunks of 24 MB
// each way, 0.70 ms for 12 + 12).  With a periodic y, stripe 0 also runs each
// shifted pass over the tile rows that the shift moves past the last row, and
// upload chunk 0 carries the rows they read.  The arithmetic, block ids and
// energy partials are those of the unstriped step, so spins and energy are bit
// for bit the same.  Applies to tiled 2D plans without the dipolar term, one
// step, pinned host memory; `used` is false otherwise.
constexpr int kPipeStripesDefault = 4;
constexpr int kPipeStreams = 3;  // uploads (the origin), downloads, compute

// The pinned mirror of the plan's status word (int at [0]) and of one energy
// (double at byte 8), written by the host-array step's last copies.
double* host_energy(mj_plan* p) { return reinterpret_cast<double*>(p->h_status + 2); }

// The y reach of the plan's stencil in rows.
int stencil_reach_y(const mj_plan* p) {
    int ry = 0;
    for (int o = 0; o < p->sp.n_off; ++o) ry = std::max(ry, std::abs(p->sp.off[o][1]));
    return ry;
}

// Stripes of the host-array step for this plan: 0 when it does not stripe.
// Each stripe is at least 2 (Q - 1) + 1 = 5 tile rows deep, so that the
// shifted ranges of every pass stay ordered.  The stencil must reach at most
// one tile row, also across a periodic y edge (a last tile row shorter than
// the reach would put two tile rows in reach of row 0).
int host_stripes(const mj_plan* p) {
    const int nty = tiled_tile_rows(p);
    const int TY = kTiledVariantTY[p->tile_variant];
    const int ry = stencil_reach_y(p);
    if (ry > TY) return 0;
    if (p->sp.periodic[1] && p->sp.L[1] - TY * (nty - 1) < ry) return 0;
    const int want = p->host_stripes > 0 ? p->host_stripes : kPipeStripesDefault;
    const int K = std::min(want, nty / 5);
    return K >= 2 ? K : 0;
}

// The striped step's work, forked from and joined back into pipe_stream[0]
// (captured once as a graph and replayed; the step index comes from the
// plan's device step counter).
mj_status striped_enqueue(mj_plan* p, double* m_host, double* m_mapped, const DynCoef& c, int energy_mode,
                          bool E_wanted) {
    const bool before = energy_mode == MJ_ENERGY_BEFORE;
    const int64_t N = p->N, Lx = p->sp.L[0], Ly = p->sp.L[1];
    const int nty = tiled_tile_rows(p);
    const int K = host_stripes(p);
    const int TY = kTiledVariantTY[p->tile_variant];
    const int ry = stencil_reach_y(p);
    const bool per_y = p->sp.periodic[1] != 0;
    // passes of the step: (pass id, stencil input, own-site m_n, output, aux, aux2, energy partials)
    struct Pass {
        int id;
        const double* ms;
        const double* mn;
        double* out;
        double* aux;
        double* aux2;
        bool energy;
    };
    double* m = p->d_tmp_m;
    double* result = m;
    std::vector<Pass> passes;
    if (c.integrator == MJ_EULER) {
        passes.push_back({1, m, nullptr, p->d_mid, nullptr, nullptr, E_wanted && before});
        result = p->d_mid;
    } else if (c.integrator == MJ_HEUN_MATJES) {
        passes.push_back({2, m, nullptr, p->d_mid, p->d_aux, p->d_aux2, E_wanted && before});
        passes.push_back({3, p->d_mid, nullptr, m, p->d_aux, p->d_aux2, false});
    } else {
        double* bstore = (c.thermal && c.noise == MJ_NOISE_PHILOX && p->store_draw) ? p->d_aux : nullptr;
        passes.push_back({4, m, nullptr, p->d_mid, bstore, nullptr, E_wanted && before});
        passes.push_back({5, p->d_mid, m, m, bstore, nullptr, false});
    }
    const int r = static_cast<int>(passes.size()) - 1;  // the pass that writes `result`
    if (E_wanted && !before) passes.push_back({0, result, nullptr, nullptr, nullptr, nullptr, true});
    const int Q = static_cast<int>(passes.size());
    // stripe k: tile rows [t[k], t[k + 1])
    std::vector<int> t(K + 1);
    for (int k = 0; k <= K; ++k) t[k] = static_cast<int>(static_cast<int64_t>(k) * nty / K);
    // the tile-row ranges of pass q in stripe k (two with a periodic wrap)
    auto ranges = [&](int q, int k, int out[2][2]) {
        const int sh = Q - 1 - q;
        int n = 0;
        const int lo = k == 0 ? 0 : t[k] + sh;
        const int hi = k == K - 1 ? nty - (per_y ? sh : 0) : t[k + 1] + sh;
        out[n][0] = lo;
        out[n++][1] = hi;
        if (k == 0 && per_y && sh > 0) {
            out[n][0] = nty - sh;
            out[n++][1] = nty;
        }
        return n;
    };
    auto row_of = [&](int tile_row) { return std::min<int64_t>(static_cast<int64_t>(tile_row) * TY, Ly); };
    // upload chunks in rows: chunk k = [u[k], u[k + 1]); with a periodic y chunk 0 also
    // holds the wrap rows [w, Ly) that the shifted first pass reads
    const int sh0 = Q - 1;
    const int64_t w = per_y ? std::max<int64_t>(0, (sh0 > 0 ? row_of(nty - sh0) : Ly) - ry) : Ly;
    std::vector<int64_t> u(K + 1);
    u[0] = 0;
    for (int k = 0; k < K; ++k) {
        int rg[2][2];
        ranges(0, k, rg);
        u[k + 1] = k == K - 1 ? w : std::min(w, std::max(u[k], row_of(rg[0][1]) + ry));
    }
    mj_status st;
    cudaStream_t sin = p->pipe_stream[0], sout = p->pipe_stream[1], sc = p->pipe_stream[2];
    cudaEvent_t* ev_in = p->pipe_events.data();
    cudaEvent_t* ev_out = ev_in + K;
    cudaEvent_t ev_fork = ev_out[K];
    cudaEvent_t* ev_join = ev_out + K + 1;
    cudaEventRecord(ev_fork, sin);
    for (int q = 1; q < kPipeStreams; ++q) cudaStreamWaitEvent(p->pipe_stream[q], ev_fork, 0);
    auto upload = [&](int64_t r0, int64_t r1) -> mj_status {
        if (r1 <= r0) return MJ_OK;
        const size_t off = static_cast<size_t>(3 * Lx * r0), cnt = static_cast<size_t>(3 * Lx * (r1 - r0));
        return cuda_status(cudaMemcpyAsync(p->d_stage + off, m_host + off, sizeof(double) * cnt, cudaMemcpyHostToDevice,
                                           sin), "striped upload");
    };
    for (int k = 0; k < K; ++k) {
        if (k == 0 && (st = upload(w, Ly)) != MJ_OK) return st;
        if ((st = upload(u[k], u[k + 1])) != MJ_OK) return st;
        cudaEventRecord(ev_in[k], sin);
    }
    for (int k = 0; k < K; ++k) {
        cudaStreamWaitEvent(sc, ev_in[k], 0);
        if (k == 0 && w < Ly && (st = aos_to_soa_range(p->d_stage, m, Lx * w, Lx * (Ly - w), N, sc)) != MJ_OK) return st;
        if (u[k + 1] > u[k] && (st = aos_to_soa_range(p->d_stage, m, Lx * u[k], Lx * (u[k + 1] - u[k]), N, sc)) != MJ_OK)
            return st;
        int down[2][2];
        int ndown = 0;
        for (int q = 0; q < Q; ++q) {
            const Pass& P = passes[q];
            int rg[2][2];
            const int n = ranges(q, k, rg);
            for (int i = 0; i < n; ++i) {
                if (rg[i][1] <= rg[i][0]) continue;
                st = launch_tiled(p, P.id, c, P.ms, P.mn, P.out, P.aux, P.aux2, DipView{}, nullptr, 0u, sc,
                                  P.energy ? 1 : 0, rg[i][0], rg[i][1] - rg[i][0]);
                if (st != MJ_OK) return st;
            }
            if (q == r) {
                ndown = n;
                for (int i = 0; i < n; ++i) {
                    down[i][0] = rg[i][0];
                    down[i][1] = rg[i][1];
                }
            }
        }
        if (m_mapped) {
            // the download stream writes the stripe's rows straight into the
            // mapped host buffer (later stripes only write other rows of `result`)
            cudaEventRecord(ev_out[k], sc);
            cudaStreamWaitEvent(sout, ev_out[k], 0);
            for (int i = 0; i < ndown; ++i) {
                const int64_t r0 = row_of(down[i][0]), r1 = row_of(down[i][1]);
                if (r1 > r0 && (st = soa_to_aos_stream(result, m_mapped, Lx * r0, Lx * (r1 - r0), N, sout)) != MJ_OK)
                    return st;
            }
            continue;
        }
        for (int i = 0; i < ndown; ++i) {
            const int64_t r0 = row_of(down[i][0]), r1 = row_of(down[i][1]);
            if (r1 > r0 && (st = soa_to_aos_range(result, p->d_stage, Lx * r0, Lx * (r1 - r0), N, sc)) != MJ_OK) return st;
        }
        cudaEventRecord(ev_out[k], sc);
        cudaStreamWaitEvent(sout, ev_out[k], 0);
        for (int i = 0; i < ndown; ++i) {
            const int64_t r0 = row_of(down[i][0]), r1 = row_of(down[i][1]);
            if (r1 <= r0) continue;
            const size_t off = static_cast<size_t>(3 * Lx * r0), cnt = static_cast<size_t>(3 * Lx * (r1 - r0));
            if ((st = cuda_status(cudaMemcpyAsync(m_host + off, p->d_stage + off, sizeof(double) * cnt,
                                                  cudaMemcpyDeviceToHost, sout), "striped download")) != MJ_OK)
                return st;
        }
    }
    // every stripe's passes (energy partials included) have run on sc before it
    // reads the status word and sums the energy
    if ((st = cuda_status(cudaMemcpyAsync(p->h_status, p->d_status, sizeof(int), cudaMemcpyDeviceToHost, sc),
                          "status mirror")) != MJ_OK)
        return st;
    if (E_wanted) {
        const int nthr = 32 * kTiledVariantBYT[p->tile_variant];
        if ((st = launch_ordered_sum(p->d_partials, static_cast<int>(tiled_energy_blocks(p)), nthr, p->d_scalar, sc)) != MJ_OK)
            return st;
        if ((st = cuda_status(cudaMemcpyAsync(host_energy(p), p->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, sc),
                              "energy mirror")) != MJ_OK)
            return st;
    }
    // join every stream back into the origin
    for (int q = 1; q < kPipeStreams; ++q) {
        cudaEventRecord(ev_join[q], p->pipe_stream[q]);
        cudaStreamWaitEvent(sin, ev_join[q], 0);
    }
    return MJ_OK;
}

mj_status step_host_striped(mj_plan* p, double* m_host, const mj_dyn_params* prm, double* E_host, bool& used) {
    used = false;
    if (!p->is_stencil || p->sp.shape == 0 || p->sp.L[2] != 1 || p->dip_on) return MJ_OK;
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, m_host) != cudaSuccess || pa.type != cudaMemoryTypeHost) {
        cudaGetLastError();  // a pageable pointer is not an error here
        return MJ_OK;
    }
    // the buffer's device address when it is mapped (kernels then write the result into it)
    double* m_mapped = p->host_zerocopy ? static_cast<double*>(pa.devicePointer) : nullptr;
    const int K = host_stripes(p);
    if (K == 0) return MJ_OK;
    DynCoef c;
    mj_status st = dyn_coef(prm, p, c);
    if (st != MJ_OK) return st;
    if ((st = ensure_host_scratch(p)) != MJ_OK) return st;
    if (!p->d_stepctr && (st = dalloc(&p->d_stepctr, 4, "step counter")) != MJ_OK) return st;
    used = true;
    c.step_base = p->d_stepctr;
    for (int q = 0; q < kPipeStreams; ++q)
        if (!p->pipe_stream[q] &&
            (st = cuda_status(cudaStreamCreateWithFlags(&p->pipe_stream[q], cudaStreamNonBlocking), "pipeline stream")) != MJ_OK)
            return st;
    // uploads, downloads, the fork, the joins, the start
    const int nev = 2 * K + 1 + kPipeStreams + 1;
    while (static_cast<int>(p->pipe_events.size()) < nev) {
        cudaEvent_t e;
        if ((st = cuda_status(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "pipeline event")) != MJ_OK) return st;
        p->pipe_events.push_back(e);
    }
    cudaStream_t sin = p->pipe_stream[0];
    // the graph holds the host pointer, the coefficients, the stencil and the kernel configuration
    std::string key(reinterpret_cast<const char*>(&c), sizeof(c));
    key += std::string(reinterpret_cast<const char*>(&p->sp), sizeof(p->sp));
    key += std::string(reinterpret_cast<const char*>(&m_host), sizeof(m_host));
    key += std::string(reinterpret_cast<const char*>(&m_mapped), sizeof(m_mapped));
    key += std::string(reinterpret_cast<const char*>(&p->d_bmap), sizeof(p->d_bmap));
    key += "/" + std::to_string(E_host != nullptr) + "/" + std::to_string(prm->energy_mode) + "/" +
           std::to_string(p->tile_variant) + "/" + std::to_string(p->store_draw) + "/" + std::to_string(K);
    if (!p->host_graph_exec || p->host_graph_key != key) {
        if (p->host_graph_exec) cudaGraphExecDestroy(p->host_graph_exec);
        p->host_graph_exec = nullptr;
        if ((st = cuda_status(cudaStreamBeginCapture(sin, cudaStreamCaptureModeThreadLocal), "begin capture")) != MJ_OK)
            return st;
        const mj_status inner = striped_enqueue(p, m_host, m_mapped, c, prm->energy_mode, E_host != nullptr);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(sin, &graph);
        if (inner != MJ_OK) {
            if (graph) cudaGraphDestroy(graph);
            return inner;
        }
        if ((st = cuda_status(e, "end capture")) != MJ_OK) return st;
        const cudaError_t ei = cudaGraphInstantiate(&p->host_graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        if ((st = cuda_status(ei, "graph instantiate")) != MJ_OK) {
            p->host_graph_exec = nullptr;
            return st;
        }
        p->host_graph_key = key;
    }
    // after the work already queued on the legacy stream: the step index, then the step
    cudaEvent_t ev_start = p->pipe_events[nev - 1];
    cudaEventRecord(ev_start, 0);
    cudaStreamWaitEvent(sin, ev_start, 0);
    if ((st = step_counter(p->d_stepctr, prm->step0, false, sin)) != MJ_OK) return st;
    if ((st = cuda_status(cudaGraphLaunch(p->host_graph_exec, sin), "graph launch")) != MJ_OK) return st;
    if ((st = cuda_status(cudaStreamSynchronize(sin), "striped step")) != MJ_OK) return st;
    if ((st = status_from_word(p, *p->h_status)) != MJ_OK) return st;
    if (E_host) *E_host = *host_energy(p);
    return MJ_OK;
}

mj_status run_steps(mj_plan* p, double* m, const mj_dyn_params* prm, int32_t nsteps, double* E_dev, cudaStream_t s) {
    if (nsteps < 0) return set_error(MJ_ERR_ARG, "nsteps must be >= 0");
    DynCoef c;
    mj_status st = dyn_coef(prm, p, c);
    if (st != MJ_OK) return st;
    return step_sequence(p, m, c, prm->energy_mode, prm->step0, nsteps, E_dev, s);
}

}  // namespace
}  // namespace mj

using namespace mj;

extern "C" {

const char* mj_last_error(void) { return g_err.c_str(); }
const char* mj_version(void) { return "matjes_b200 0.1 (sm_100a, fp64)"; }

mj_status mj_plan_create(const mj_lattice_desc* lat, const mj_hamiltonian_desc* ham, int32_t device, mj_plan** out) {
    if (!lat || !ham || !out) return set_error(MJ_ERR_ARG, "null argument");
    *out = nullptr;
    if ((ham->nJ > 0 && !ham->J) || (ham->nD > 0 && !ham->D) || (ham->nK > 0 && !ham->K) || ham->nJ < 0 ||
        ham->nD < 0 || ham->nK < 0)
        return set_error(MJ_ERR_ARG, "term count without term array");
    mj_status st = cuda_status(cudaSetDevice(device), "cudaSetDevice");
    if (st != MJ_OK) return st;
    Geometry g;
    std::string err;
    if (!build_geometry(*lat, g, err)) return set_error(MJ_ERR_ARG, err);
    std::vector<Block> blocks;
    std::vector<double> onsite;
    if (!build_blocks(g, *ham, blocks, onsite, err)) return set_error(MJ_ERR_GEOMETRY, err);
    mj_plan* p = new mj_plan();
    p->device = device;
    p->nmag = g.nmag;
    p->ncell = static_cast<int64_t>(lat->L[0]) * lat->L[1] * lat->L[2];
    p->N = p->ncell * g.nmag;
    p->blocks = blocks;
    p->geom = g;
    p->ham = *ham;
    p->ham.J = nullptr;
    p->ham.D = nullptr;
    p->ham.K = nullptr;
    p->termJ.assign(ham->J, ham->J + ham->nJ);
    p->termD.assign(ham->D, ham->D + ham->nD);
    p->termK.assign(ham->K, ham->K + ham->nK);
    const bool zee_on = ham->zeeman_on ||
                        std::sqrt(ham->B_ext[0] * ham->B_ext[0] + ham->B_ext[1] * ham->B_ext[1] + ham->B_ext[2] * ham->B_ext[2]) >= 1e-8;
    StencilParams& sp = p->sp;
    std::memset(&sp, 0, sizeof(sp));
    for (int d = 0; d < 3; ++d) {
        sp.L[d] = lat->L[d];
        sp.periodic[d] = lat->periodic[d] ? 1 : 0;
    }
    sp.zee_on = zee_on ? 1 : 0;
    for (int k = 0; k < 3; ++k) sp.bext[k] = ham->B_ext[k];
    p->bext_cell.assign(ham->B_ext, ham->B_ext + 3);
    p->is_stencil = g.nmag == 1 && make_stencil(blocks, onsite, sp);
    if (p->is_stencil) {
        match_shape(sp);
        p->tiled_shape = sp.shape;
    }
    if (p->is_stencil) {
        sp.zc = -((1.0 * kMuB * ham->c_zeeman) * lat->moment[g.magatom[0]]);
    } else {
        if (ham->dip_on) {
            free_plan(p);
            return set_error(MJ_ERR_UNSUPPORTED, "the FFT dipolar term needs one magnetic atom per cell");
        }
        if ((st = ell_from_blocks(p, g, blocks, onsite)) != MJ_OK) {
            free_plan(p);
            return st;
        }
        if (zee_on) {
            std::vector<double> zc(p->N);
            for (int64_t s2 = 0; s2 < p->N; ++s2) zc[s2] = -((1.0 * kMuB * ham->c_zeeman) * lat->moment[g.magatom[s2 % g.nmag]]);
            if ((st = dalloc(&p->d_zee, p->N, "zeeman")) != MJ_OK ||
                (st = cuda_status(cudaMemcpy(p->d_zee, zc.data(), sizeof(double) * p->N, cudaMemcpyHostToDevice), "zeeman upload")) != MJ_OK) {
                free_plan(p);
                return st;
            }
        }
    }
    if ((st = alloc_scratch(p)) != MJ_OK) {
        free_plan(p);
        return st;
    }
    if (ham->dip_on) {
        std::vector<double> K;
        if (!build_dipolar_kernel(g, *ham, p->nrep, K, err)) {
            free_plan(p);
            return set_error(MJ_ERR_UNSUPPORTED, err);
        }
        p->dip_on = true;
        if ((st = dipolar_create(p, K, 0)) != MJ_OK) {
            p->dip_on = false;
            free_plan(p);
            return st;
        }
    }
    if ((st = cuda_status(cudaDeviceSynchronize(), "plan create")) != MJ_OK) {
        free_plan(p);
        return st;
    }
    *out = p;
    return MJ_OK;
}

mj_status mj_stencil_describe(const mj_lattice_desc* lat, const mj_hamiltonian_desc* ham, int32_t cap, int32_t* n_off,
                              int32_t* offsets, double* W, double* W0, double* zc) {
    if (!lat || !ham || !n_off || (cap > 0 && (!offsets || !W)) || !W0 || !zc) return set_error(MJ_ERR_ARG, "null argument");
    Geometry g;
    std::string err;
    if (!build_geometry(*lat, g, err)) return set_error(MJ_ERR_ARG, err);
    std::vector<Block> blocks;
    std::vector<double> onsite;
    if (!build_blocks(g, *ham, blocks, onsite, err)) return set_error(MJ_ERR_GEOMETRY, err);
    if (g.nmag != 1) return set_error(MJ_ERR_UNSUPPORTED, "multi-atom cells compile to an ELL matrix, not a stencil");
    StencilParams sp;
    std::memset(&sp, 0, sizeof(sp));
    if (!make_stencil(blocks, onsite, sp)) return set_error(MJ_ERR_UNSUPPORTED, "more neighbour offsets than kMaxOff");
    *n_off = sp.n_off;
    if (sp.n_off > cap) return set_error(MJ_ERR_ARG, "offset capacity too small");
    for (int k = 0; k < sp.n_off; ++k) {
        for (int d = 0; d < 3; ++d) offsets[3 * k + d] = sp.off[k][d];
        for (int q = 0; q < 9; ++q) W[9 * k + q] = sp.W[k][q];
    }
    for (int q = 0; q < 9; ++q) W0[q] = sp.W0[q];
    *zc = -((1.0 * kMuB * ham->c_zeeman) * lat->moment[g.magatom[0]]);
    return MJ_OK;
}

mj_status mj_plan_from_coo(int64_t nsites, int64_t nnz, const int64_t* rows, const int64_t* cols, const double* vals,
                           int32_t base, const double* zeeman, const double* b_cell, int32_t device, mj_plan** out) {
    if (!out || nsites <= 0 || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals)) || (base != 0 && base != 1))
        return set_error(MJ_ERR_ARG, "bad COO arguments");
    *out = nullptr;
    mj_status st = cuda_status(cudaSetDevice(device), "cudaSetDevice");
    if (st != MJ_OK) return st;
    // group the scalar triplets into 3x3 site blocks H_st
    std::vector<Entry> blk;
    blk.reserve(static_cast<size_t>(nnz));
    for (int64_t k = 0; k < nnz; ++k) {
        const int64_t r = rows[k] - base, c = cols[k] - base;
        if (r < 0 || c < 0 || r >= 3 * nsites || c >= 3 * nsites) return set_error(MJ_ERR_ARG, "COO index out of range");
        Entry e;
        e.row = r / 3;
        e.col = c / 3;
        std::fill(e.W, e.W + 9, 0.0);
        e.W[3 * (r % 3) + (c % 3)] = vals[k];
        blk.push_back(e);
    }
    std::sort(blk.begin(), blk.end(), [](const Entry& a, const Entry& b) {
        return a.row != b.row ? a.row < b.row : a.col < b.col;
    });
    std::vector<Entry> H;
    for (const Entry& e : blk) {
        if (!H.empty() && H.back().row == e.row && H.back().col == e.col) {
            for (int q = 0; q < 9; ++q) H.back().W[q] += e.W[q];
        } else {
            H.push_back(e);
        }
    }
    mj_plan* p = new mj_plan();
    p->device = device;
    p->nmag = 1;
    p->ncell = nsites;
    p->N = nsites;
    p->is_stencil = false;
    std::vector<Entry> ent;
    for (const Entry& e : H) push_pair(ent, e.row, e.col, e.W);
    if ((st = make_ell(p, ent)) != MJ_OK) {
        free_plan(p);
        return st;
    }
    if (zeeman) {
        std::vector<double> zc(nsites);
        for (int64_t s = 0; s < nsites; ++s) zc[s] = -zeeman[s];
        if ((st = dalloc(&p->d_zee, nsites, "zeeman")) != MJ_OK ||
            (st = cuda_status(cudaMemcpy(p->d_zee, zc.data(), sizeof(double) * nsites, cudaMemcpyHostToDevice), "zeeman")) != MJ_OK) {
            free_plan(p);
            return st;
        }
        p->bext_cell.assign(3, 0.0);
        if (b_cell) {
            std::vector<double> soa(3 * nsites);
            for (int64_t s = 0; s < nsites; ++s)
                for (int k = 0; k < 3; ++k) soa[k * nsites + s] = b_cell[3 * s + k];
            if ((st = dalloc(&p->d_bmap, 3 * nsites, "bmap")) != MJ_OK ||
                (st = cuda_status(cudaMemcpy(p->d_bmap, soa.data(), sizeof(double) * 3 * nsites, cudaMemcpyHostToDevice), "bmap")) != MJ_OK) {
                free_plan(p);
                return st;
            }
        }
    }
    if ((st = alloc_scratch(p)) != MJ_OK) {
        free_plan(p);
        return st;
    }
    *out = p;
    return MJ_OK;
}

mj_status mj_plan_destroy(mj_plan* plan) {
    if (!plan) return MJ_OK;
    cudaSetDevice(plan->device);
    free_plan(plan);
    return MJ_OK;
}

mj_status mj_plan_nsites(const mj_plan* plan, int64_t* n) {
    if (!plan || !n) return set_error(MJ_ERR_ARG, "null argument");
    *n = plan->N;
    return MJ_OK;
}

mj_status mj_plan_noffsets(const mj_plan* plan, int32_t* n) {
    if (!plan || !n) return set_error(MJ_ERR_ARG, "null argument");
    *n = plan->is_stencil ? plan->sp.n_off : 0;
    return MJ_OK;
}

mj_status mj_plan_set_variant(mj_plan* plan, int32_t variant) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    if (variant < -1 || variant >= kTiledVariants) return set_error(MJ_ERR_ARG, "variant must be -1..5");
    if (variant >= 0 && !(plan->is_stencil && plan->tiled_shape != 0))
        return set_error(MJ_ERR_UNSUPPORTED, "no tiled kernel for this plan's offsets");
    if (variant < 0) {
        plan->sp.shape = 0;
    } else {
        plan->sp.shape = plan->tiled_shape;
        plan->tile_variant = variant;
    }
    if (plan->graph_exec) {  // the captured graph holds the old kernels
        cudaGraphExecDestroy(plan->graph_exec);
        plan->graph_exec = nullptr;
        plan->graph_key.clear();
    }
    return MJ_OK;
}

mj_status mj_plan_autotune(mj_plan* plan, const double* m, const mj_dyn_params* prm, int32_t steps, int32_t* best,
                           int32_t* best_tma, double* ms_per_step) {
    if (!plan || !m || !prm || !best || steps < 1) return set_error(MJ_ERR_ARG, "bad autotune arguments");
    cudaSetDevice(plan->device);
    mj_status st = ensure_host_scratch(plan);
    if (st != MJ_OK) return st;
    DynCoef c;
    if ((st = dyn_coef(prm, plan, c)) != MJ_OK) return st;
    const int32_t v0 = (plan->is_stencil && plan->sp.shape != 0) ? plan->tile_variant : -1;
    const bool has_tiled = plan->is_stencil && plan->tiled_shape != 0;
    cudaEvent_t a, b;
    if ((st = cuda_status(cudaEventCreate(&a), "event")) != MJ_OK) return st;
    if ((st = cuda_status(cudaEventCreate(&b), "event")) != MJ_OK) {
        cudaEventDestroy(a);
        return st;
    }
    double best_ms = 1e300;
    int32_t best_v = v0;
    bool best_t = plan->use_tma;
    // configurations: 0 generic, 1..6 tiled variants 0..5 with plain loads, 7..12 with TMA
    for (int cfg = 0; cfg < 1 + 2 * kTiledVariants; ++cfg) {
        const int32_t v = cfg == 0 ? -1 : (cfg - 1) % kTiledVariants;
        const bool tma = cfg > kTiledVariants;
        double ms = -1.0;
        if ((v >= 0 && !has_tiled) || (v == -1 && !plan->is_stencil)) {
            if (ms_per_step) ms_per_step[cfg] = ms;
            continue;
        }
        plan->use_tma = tma;
        if (plan->is_stencil && (st = mj_plan_set_variant(plan, v)) != MJ_OK) break;
        if ((st = cuda_status(cudaMemcpy(plan->d_tmp_m, m, sizeof(double) * 3 * plan->N, cudaMemcpyDeviceToDevice),
                              "autotune copy")) != MJ_OK)
            break;
        if ((st = step_sequence(plan, plan->d_tmp_m, c, MJ_ENERGY_BEFORE, prm->step0, 1, nullptr, 0)) != MJ_OK) break;
        cudaEventRecord(a, 0);
        if ((st = step_sequence(plan, plan->d_tmp_m, c, MJ_ENERGY_BEFORE, prm->step0, steps, nullptr, 0)) != MJ_OK) break;
        cudaEventRecord(b, 0);
        if ((st = cuda_status(cudaEventSynchronize(b), "autotune sync")) != MJ_OK) break;
        float f = 0.0f;
        cudaEventElapsedTime(&f, a, b);
        ms = f / steps;
        if (ms_per_step) ms_per_step[cfg] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best_v = v;
            best_t = tma;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (st != MJ_OK) return st;
    plan->use_tma = best_t;
    if (plan->is_stencil && (st = mj_plan_set_variant(plan, best_v)) != MJ_OK) return st;
    if ((st = mj_plan_check_status(plan)) != MJ_OK) return st;
    *best = best_v;
    if (best_tma) *best_tma = best_t ? 1 : 0;
    return MJ_OK;
}

mj_status mj_plan_set_tma(mj_plan* plan, int32_t enable) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    plan->use_tma = enable != 0;
    if (plan->graph_exec) {
        cudaGraphExecDestroy(plan->graph_exec);
        plan->graph_exec = nullptr;
        plan->graph_key.clear();
    }
    return MJ_OK;
}

mj_status mj_plan_set_option(mj_plan* plan, int32_t option, int32_t value) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    switch (option) {
        case MJ_OPT_TMA: plan->use_tma = value != 0; break;
        case MJ_OPT_FUSED: plan->fused_sib = value != 0; break;
        case MJ_OPT_PDL: plan->use_pdl = value != 0; break;
        case MJ_OPT_STORE_DRAW: plan->store_draw = value != 0; break;
        case MJ_OPT_HOST_STRIPES:
            if (value < 0 || value > 64) return set_error(MJ_ERR_ARG, "host stripes must be in [0, 64]");
            plan->host_stripes = value;
            break;
        case MJ_OPT_DIP_ZCONV: plan->dip_zconv = value != 0; break;
        case MJ_OPT_HOST_ZEROCOPY: plan->host_zerocopy = value != 0; break;
        case MJ_OPT_BLOCKS_PER_SM: {
            if (value != 0 && (value < 4 || value > 32))
                return set_error(MJ_ERR_ARG, "blocks per SM must be 0 or in [4, 32]");
            plan->blocks_per_sm = value;
            plan->smem_cap_bytes = 0;
            if (value > 0) {
                // enough shared memory per block that value + 1 blocks do not fit
                // on an SM and value blocks do (below the 48 KB default limit)
                cudaDeviceProp prop;
                mj_status st = cuda_status(cudaGetDeviceProperties(&prop, plan->device), "device properties");
                if (st != MJ_OK) return st;
                const size_t per_sm = prop.sharedMemPerMultiprocessor, rsv = prop.reservedSharedMemPerBlock;
                size_t b = per_sm / static_cast<size_t>(value + 1) - rsv + 128;
                b = (b + 127) / 128 * 128;
                if (b > 48 * 1024 || static_cast<size_t>(value) * (b + rsv + 1024) > per_sm)
                    return set_error(MJ_ERR_ARG, "blocks per SM: no shared memory size gives this cap");
                plan->smem_cap_bytes = static_cast<int>(b);
            }
            break;
        }
        default: return set_error(MJ_ERR_ARG, "unknown plan option " + std::to_string(option));
    }
    drop_graph(plan);
    return MJ_OK;
}

mj_status mj_plan_set_fused(mj_plan* plan, int32_t enable) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    plan->fused_sib = enable != 0;
    drop_graph(plan);
    return MJ_OK;
}

mj_status mj_plan_check_status(mj_plan* plan) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    cudaSetDevice(plan->device);
    int word = 0;
    mj_status st = cuda_status(cudaDeviceSynchronize(), "status sync");
    if (st != MJ_OK) return st;
    if ((st = cuda_status(cudaMemcpy(&word, plan->d_status, sizeof(int), cudaMemcpyDeviceToHost), "status read")) != MJ_OK)
        return st;
    return status_from_word(plan, word);
}

mj_status mj_plan_get_variant(const mj_plan* plan, int32_t* variant, int32_t* shape) {
    if (!plan || !variant || !shape) return set_error(MJ_ERR_ARG, "null argument");
    *variant = (plan->is_stencil && plan->sp.shape != 0) ? plan->tile_variant : -1;
    *shape = plan->tiled_shape;
    return MJ_OK;
}

mj_status mj_plan_set_bfield(mj_plan* plan, const double* b) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    cudaSetDevice(plan->device);
    if (!b) {
        cudaFree(plan->d_bmap);
        plan->d_bmap = nullptr;
        return MJ_OK;
    }
    const int64_t nc = plan->ncell;
    std::vector<double> soa(3 * nc);
    for (int64_t c = 0; c < nc; ++c)
        for (int k = 0; k < 3; ++k) soa[k * nc + c] = b[3 * c + k];
    mj_status st;
    if (!plan->d_bmap && (st = dalloc(&plan->d_bmap, 3 * nc, "bmap")) != MJ_OK) return st;
    if (plan->is_stencil) plan->sp.zee_on = 1;
    return cuda_status(cudaMemcpy(plan->d_bmap, soa.data(), sizeof(double) * 3 * nc, cudaMemcpyHostToDevice), "bmap upload");
}

mj_status mj_plan_set_bfield_device(mj_plan* plan, const double* b, void* stream) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    if (!b) return mj_plan_set_bfield(plan, nullptr);
    cudaSetDevice(plan->device);
    mj_status st;
    if (!plan->d_bmap && (st = dalloc(&plan->d_bmap, 3 * plan->ncell, "bmap")) != MJ_OK) return st;
    if (plan->is_stencil) plan->sp.zee_on = 1;
    return cuda_status(cudaMemcpyAsync(plan->d_bmap, b, sizeof(double) * 3 * plan->ncell, cudaMemcpyDeviceToDevice,
                                       static_cast<cudaStream_t>(stream)),
                       "bmap copy");
}

mj_status mj_state_create(const mj_plan* plan, mj_state** out) {
    if (!plan || !out) return set_error(MJ_ERR_ARG, "null argument");
    *out = nullptr;
    cudaSetDevice(plan->device);
    mj_state* s = new mj_state();
    s->plan = plan;
    mj_status st = dalloc(&s->d_m, 3 * plan->N, "state");
    if (st != MJ_OK) {
        delete s;
        return st;
    }
    cudaMemset(s->d_m, 0, sizeof(double) * 3 * plan->N);
    *out = s;
    return MJ_OK;
}

mj_status mj_state_destroy(mj_state* st) {
    if (!st) return MJ_OK;
    cudaSetDevice(st->plan->device);
    cudaFree(st->d_m);
    delete st;
    return MJ_OK;
}

mj_status mj_state_upload(mj_state* s, const double* m, void* stream) {
    if (!s || !m) return set_error(MJ_ERR_ARG, "null argument");
    mj_plan* p = const_cast<mj_plan*>(s->plan);
    cudaSetDevice(p->device);
    mj_status st = ensure_host_scratch(p);
    if (st != MJ_OK) return st;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    if ((st = cuda_status(cudaMemcpyAsync(p->d_stage, m, sizeof(double) * 3 * p->N, cudaMemcpyHostToDevice, cs), "upload")) != MJ_OK)
        return st;
    return aos_to_soa(p->d_stage, s->d_m, p->N, cs);
}

mj_status mj_state_download(const mj_state* s, double* m, void* stream) {
    if (!s || !m) return set_error(MJ_ERR_ARG, "null argument");
    mj_plan* p = const_cast<mj_plan*>(s->plan);
    cudaSetDevice(p->device);
    mj_status st = ensure_host_scratch(p);
    if (st != MJ_OK) return st;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    if ((st = soa_to_aos(s->d_m, p->d_stage, p->N, cs)) != MJ_OK) return st;
    if ((st = cuda_status(cudaMemcpyAsync(m, p->d_stage, sizeof(double) * 3 * p->N, cudaMemcpyDeviceToHost, cs), "download")) != MJ_OK)
        return st;
    return cuda_status(cudaStreamSynchronize(cs), "download sync");
}

mj_status mj_state_device_ptr(const mj_state* s, double** m) {
    if (!s || !m) return set_error(MJ_ERR_ARG, "null argument");
    *m = s->d_m;
    return MJ_OK;
}

mj_status mj_field_dev(mj_plan* plan, const double* m, double* B, double* e_site, void* stream) {
    if (!plan || !m) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(plan->device);
    return launch_field(plan, m, B, e_site, nullptr, static_cast<cudaStream_t>(stream));
}

mj_status mj_field(mj_plan* plan, const mj_state* s, double* B, double* e_site, void* stream) {
    if (!s) return set_error(MJ_ERR_ARG, "null state");
    return mj_field_dev(plan, s->d_m, B, e_site, stream);
}

mj_status mj_energy(mj_plan* plan, const mj_state* s, double* E) {
    if (!plan || !s || !E) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(plan->device);
    mj_status st = launch_energy(plan, s->d_m, plan->d_scalar, 0);
    if (st != MJ_OK) return st;
    return cuda_status(cudaMemcpy(E, plan->d_scalar, sizeof(double), cudaMemcpyDeviceToHost), "energy");
}

mj_status mj_field_host(mj_plan* plan, const double* m, double* B, double* e_site) {
    if (!plan || !m || !B) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(plan->device);
    mj_status st = ensure_host_scratch(plan);
    if (st != MJ_OK) return st;
    const int64_t N = plan->N;
    if ((st = cuda_status(cudaMemcpy(plan->d_stage, m, sizeof(double) * 3 * N, cudaMemcpyHostToDevice), "upload")) != MJ_OK) return st;
    if ((st = aos_to_soa(plan->d_stage, plan->d_tmp_m, N, 0)) != MJ_OK) return st;
    if ((st = launch_field(plan, plan->d_tmp_m, plan->d_tmp_b, e_site ? plan->d_tmp_e : nullptr, nullptr, 0)) != MJ_OK) return st;
    if ((st = soa_to_aos(plan->d_tmp_b, plan->d_stage, N, 0)) != MJ_OK) return st;
    if ((st = cuda_status(cudaMemcpy(B, plan->d_stage, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost), "download B")) != MJ_OK) return st;
    if (e_site && (st = cuda_status(cudaMemcpy(e_site, plan->d_tmp_e, sizeof(double) * N, cudaMemcpyDeviceToHost), "download e")) != MJ_OK)
        return st;
    return MJ_OK;
}

mj_status mj_step_dev(mj_plan* plan, double* m, const mj_dyn_params* prm, int32_t nsteps, double* E_dev, void* stream) {
    if (!plan || !m) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(plan->device);
    return run_steps(plan, m, prm, nsteps, E_dev, static_cast<cudaStream_t>(stream));
}

mj_status mj_step(mj_plan* plan, mj_state* s, const mj_dyn_params* prm, int32_t nsteps, double* E_dev, void* stream) {
    if (!s) return set_error(MJ_ERR_ARG, "null state");
    return mj_step_dev(plan, s->d_m, prm, nsteps, E_dev, stream);
}

mj_status mj_step_host(mj_plan* plan, double* m, const mj_dyn_params* prm, int32_t nsteps, double* E_host) {
    if (!plan || !m) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(plan->device);
    mj_status st;
    if (nsteps == 1) {  // one step from pinned host memory: copies and passes overlapped by stripes
        bool used = false;
        if ((st = step_host_striped(plan, m, prm, E_host, used)) != MJ_OK || used) return st;
    }
    st = ensure_host_scratch(plan);
    if (st != MJ_OK) return st;
    const int64_t N = plan->N;
    double* dE = nullptr;
    if (E_host && nsteps > 0 && (st = dalloc(&dE, static_cast<size_t>(nsteps), "energies")) != MJ_OK) return st;
    if ((st = cuda_status(cudaMemcpy(plan->d_stage, m, sizeof(double) * 3 * N, cudaMemcpyHostToDevice), "upload")) == MJ_OK &&
        (st = aos_to_soa(plan->d_stage, plan->d_tmp_m, N, 0)) == MJ_OK &&
        (st = run_steps(plan, plan->d_tmp_m, prm, nsteps, dE, 0)) == MJ_OK &&
        (st = soa_to_aos(plan->d_tmp_m, plan->d_stage, N, 0)) == MJ_OK &&
        (st = cuda_status(cudaMemcpy(m, plan->d_stage, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost), "download")) == MJ_OK &&
        (st = cuda_status(cudaMemcpy(plan->h_status, plan->d_status, sizeof(int), cudaMemcpyDeviceToHost), "status")) ==
            MJ_OK &&
        (st = status_from_word(plan, *plan->h_status)) == MJ_OK && dE) {
        st = cuda_status(cudaMemcpy(E_host, dE, sizeof(double) * nsteps, cudaMemcpyDeviceToHost), "energies");
    }
    cudaFree(dE);
    return st;
}

mj_status mj_graph_run(mj_plan* plan, mj_state* s, const mj_dyn_params* prm, int32_t nsteps, int32_t nreplay,
                       double* E_dev, void* stream) {
    if (!plan || !s || !prm || nsteps < 1 || nreplay < 0) return set_error(MJ_ERR_ARG, "bad graph arguments");
    cudaSetDevice(plan->device);
    DynCoef c;
    mj_status st = dyn_coef(prm, plan, c);
    if (st != MJ_OK) return st;
    if (!plan->d_stepctr && (st = dalloc(&plan->d_stepctr, 4, "step counter")) != MJ_OK) return st;
    if (!plan->cap_stream &&
        (st = cuda_status(cudaStreamCreateWithFlags(&plan->cap_stream, cudaStreamNonBlocking), "capture stream")) != MJ_OK)
        return st;
    c.step_base = plan->d_stepctr;
    // the captured graph depends on the state pointer, the coefficients and the step count
    std::string key(reinterpret_cast<const char*>(&c), sizeof(c));
    key += std::string(reinterpret_cast<const char*>(&s->d_m), sizeof(s->d_m));
    key += std::string(reinterpret_cast<const char*>(&E_dev), sizeof(E_dev));
    key += std::to_string(nsteps) + "/" + std::to_string(prm->energy_mode);
    if (!plan->graph_exec || plan->graph_key != key) {
        if (plan->graph_exec) {
            cudaGraphExecDestroy(plan->graph_exec);
            plan->graph_exec = nullptr;
        }
        cudaStream_t cs = plan->cap_stream;
        if ((st = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture")) != MJ_OK)
            return st;
        const bool prof = plan->prof_on;
        plan->prof_on = false;  // no event records inside a graph
        mj_status inner = step_sequence(plan, s->d_m, c, prm->energy_mode, 0u, nsteps, E_dev, cs);
        plan->prof_on = prof;
        if (inner == MJ_OK) inner = step_counter(plan->d_stepctr, static_cast<uint32_t>(nsteps), true, cs);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(cs, &graph);
        if (inner != MJ_OK) {
            if (graph) cudaGraphDestroy(graph);
            return inner;
        }
        if ((st = cuda_status(e, "end capture")) != MJ_OK) return st;
        e = cudaGraphInstantiate(&plan->graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        if ((st = cuda_status(e, "graph instantiate")) != MJ_OK) {
            plan->graph_exec = nullptr;
            return st;
        }
        plan->graph_key = key;
    }
    cudaStream_t us = static_cast<cudaStream_t>(stream);
    if ((st = step_counter(plan->d_stepctr, prm->step0, false, us)) != MJ_OK) return st;
    for (int32_t r = 0; r < nreplay; ++r)
        if ((st = cuda_status(cudaGraphLaunch(plan->graph_exec, us), "graph launch")) != MJ_OK) return st;
    return MJ_OK;
}

mj_status mj_profile_enable(mj_plan* plan, int32_t enable) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    cudaSetDevice(plan->device);
    prof_clear(plan);
    plan->prof_on = enable != 0;
    return MJ_OK;
}

mj_status mj_profile_read(mj_plan* plan, int32_t cap, char* names, double* total_ms, int64_t* launches, int32_t* n) {
    if (!plan || !n || (cap > 0 && (!names || !total_ms || !launches))) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(plan->device);
    mj_status st = cuda_status(cudaDeviceSynchronize(), "profile sync");
    if (st != MJ_OK) return st;
    const int k = static_cast<int>(plan->prof_names.size());
    *n = k;
    std::vector<double> tot(k, 0.0);
    std::vector<int64_t> cnt(k, 0);
    for (auto& r : plan->prof) {
        float ms = 0.0f;
        if ((st = cuda_status(cudaEventElapsedTime(&ms, r.a, r.b), "event elapsed")) != MJ_OK) return st;
        tot[r.id] += ms;
        cnt[r.id] += 1;
    }
    for (int i = 0; i < k && i < cap; ++i) {
        std::memset(names + 32 * i, 0, 32);
        std::strncpy(names + 32 * i, plan->prof_names[i].c_str(), 31);
        total_ms[i] = tot[i];
        launches[i] = cnt[i];
    }
    return MJ_OK;
}

mj_status mj_measure_temperature(mj_plan* plan, const mj_state* s, double* T) {
    if (!plan || !s || !T) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(plan->device);
    mj_status st = launch_temperature(plan, s->d_m, plan->d_scalar, 0);
    if (st != MJ_OK) return st;
    double v[2];
    if ((st = cuda_status(cudaMemcpy(v, plan->d_scalar, sizeof(v), cudaMemcpyDeviceToHost), "temperature")) != MJ_OK) return st;
    *T = v[0] / v[1] / 2.0 / kKB;
    return MJ_OK;
}

mj_status mj_philox_normals(uint64_t seed, uint32_t step, uint32_t stream_id, int64_t n, double* out, void* stream) {
    if (!out || n < 0) return set_error(MJ_ERR_ARG, "bad argument");
    return launch_philox(seed, step, stream_id, n, out, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
