// Metropolis Monte Carlo on the device (Metropolis-MC/MCstep.f90).
//
// The reference makes single-spin moves at random sites (choose_spin.f90), each
// a proposal and the Metropolis test of MCstep.f90:75-89 (accepted when dE < 0
// or when a uniform is below exp(max(-dE/kT, -200))).  Here a sweep moves every
// site once, colour by colour with a colouring in which no coupling joins two
// sites of one colour, so the moves of a colour are independent and run in
// parallel: the same single-spin moves and acceptance rule in another site
// order.  Two families of colourings are searched and the one with fewer
// colours kept: linear, colour (x + b y + c z) mod q (2 colours for square and
// cubic nearest neighbours, 3 for triangular), and product, colour (x mod cx,
// y mod cy, z mod cz); a periodic size must keep the colour of its wrapped
// images.  The uniforms are Philox4x32-10 draws, counter (site, sweep, stream,
// 0x4D43) under key `seed`: words 0 and 1 drive the proposal, word 2 the
// acceptance test, each turned into a uniform in (0, 1) as (w + 0.5) 2^-32.
// Proposals (track_value.f90 sample_*): the cone of sphereft (paratemp-MC/
// sampling.f90:9-62), the Ising flip, under- and over-relaxation from the
// site's field (relaxationtype.f90).  The energy change of a move is that of
// energy_single:
//   dE = -(s' - s).P - (s'^T W0 s' - s^T W0 s)/2 - (s' - s).(zc b)
// with P the pair field of the neighbours and W0 the on-site tensor.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mj_device.cuh"
#include "mj_internal.hpp"
#include "mj_stencil.cuh"

namespace mj {
namespace {

constexpr uint32_t kMcTag = 0x4D43u;  // "MC"

struct McCoef {
    double kT;          // eV
    double cos_cone;
    int proposal;       // MJ_MC_CONE or MJ_MC_ISING
    uint32_t keys[20];  // Philox round keys of the seed
    uint32_t sweep;
    uint32_t stream;
};

__device__ __forceinline__ double u32_open(uint32_t w) { return (static_cast<double>(w) + 0.5) * (1.0 / 4294967296.0); }

// sphereft: a direction in the cone of half-angle `cone` about s
__device__ __forceinline__ double3 cone_proposal(double3 s, double cos_cone, double u1, double u2) {
    const double ct = u1 + cos_cone * (1.0 - u1);
    const double st = sqrt(1.0 - ct * ct);
    const double phi = 2.0 * kPi * u2;
    const double cti = s.z;
    const double rxy2 = s.x * s.x + s.y * s.y;
    const double sti = sqrt(rxy2);
    double cpi = 1.0, spi = 0.0;
    if (!(rxy2 < 0.00001)) {
        cpi = s.x / sqrt(rxy2);
        spi = s.y / sqrt(rxy2);
    }
    const double cph = cos(phi), sph = sin(phi);
    const double t = st * sph * cti + ct * sti;
    const double3 n = make_double3(-st * cph * spi + t * cpi, st * cph * cpi + t * spi, -st * sph * sti + ct * cti);
    const double nn = sqrt(dot(n, n));
    return make_double3(n.x / nn, n.y / nn, n.z / nn);
}

// pair field P_i = sum_o W_o m_{i+o} (no on-site term)
__device__ __forceinline__ double3 pair_field(const StencilParams& P, const double* __restrict__ m, int64_t N, int x,
                                              int y, int z) {
    double3 b = make_double3(0.0, 0.0, 0.0);
    for (int k = 0; k < P.n_off; ++k) {
        int64_t j;
        if (!neighbour(P, x, y, z, k, j)) continue;
        b = mat3(P.W[k], ld3(m, j, N), b);
    }
    return b;
}

__device__ __forceinline__ double onsite_energy(const StencilParams& P, double3 s) {
    if (!P.has_onsite) return 0.0;
    return -0.5 * dot(s, mat3(P.W0, s, make_double3(0.0, 0.0, 0.0)));
}

// the proposal of a move (track_value.f90 sample_*); B the site's effective field
// -dE/dm (relaxationtype.f90 under- and over-relaxation)
__device__ __forceinline__ double3 propose(int proposal, double3 s, double3 B, double cos_cone, const uint32_t c[4]) {
    if (proposal == MJ_MC_ISING) return make_double3(-s.x, -s.y, -s.z);
    if (proposal == MJ_MC_CONE) return cone_proposal(s, cos_cone, u32_open(c[0]), u32_open(c[1]));
    const double sb = dot(s, B);
    double3 n;
    if (proposal == MJ_MC_UNDERRELAX) n = make_double3(s.x * (1.0 - sb) + B.x, s.y * (1.0 - sb) + B.y, s.z * (1.0 - sb) + B.z);
    else n = make_double3(B.x - s.x * (1.0 + sb), B.y - s.y * (1.0 + sb), B.z - s.z * (1.0 + sb));
    const double nn = sqrt(dot(n, n));
    return make_double3(n.x / nn, n.y / nn, n.z / nn);
}

// One colour class of a sweep: the sites y = ry + sy ty, z = rz + sz tz,
// x = ((k - b y - c z) mod qx) + qx tx.  A linear colouring (q, b, c) has
// qx = q, sy = sz = 1, colour k; a product colouring (cx, cy, cz) has qx = cx,
// sy = cy, sz = cz, b = c = 0 and colour (k, ry, rz).
struct McClass {
    int qx, sy, sz, b, c, k, ry, rz;
};

__global__ void __launch_bounds__(256) k_mc_color(const __grid_constant__ StencilParams P, const double* __restrict__ bmap,
                                                  double* m, const McCoef C, const McClass K,
                                                  unsigned long long* accepted) {
    const int y = K.ry + K.sy * static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    const int z = K.rz + K.sz * static_cast<int>(blockIdx.z);
    const int x0 = ((K.k - K.b * y - K.c * z) % K.qx + K.qx) % K.qx;
    const int x = x0 + K.qx * static_cast<int>(blockIdx.x * 32 + threadIdx.x);
    bool acc = false;
    if (x < P.L[0] && y < P.L[1] && z < P.L[2]) {
        const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
        const int64_t i = x + static_cast<int64_t>(P.L[0]) * (y + static_cast<int64_t>(P.L[1]) * z);
        uint32_t c[4] = {static_cast<uint32_t>(i), C.sweep, C.stream, kMcTag};
        philox10k(c, C.keys);
        const double3 s = ld3(m, i, N);
        const double3 Pf = pair_field(P, m, N, x, y, z);
        const double3 zb = zeeman(P, bmap, i, N);
        double3 B = add3(Pf, zb);
        if (P.has_onsite) B = mat3(P.W0, s, B);
        const double3 sn = propose(C.proposal, s, B, C.cos_cone, c);
        const double3 d = make_double3(sn.x - s.x, sn.y - s.y, sn.z - s.z);
        const double dE = -dot(d, Pf) + (onsite_energy(P, sn) - onsite_energy(P, s)) - dot(d, zb);
        acc = dE < 0.0;
        if (!acc && C.kT > 0.0) acc = u32_open(c[2]) < exp(fmax(-dE / C.kT, -200.0));
        if (acc) st3(m, i, N, sn);
    }
    // accepted moves of the block, added once per block (an integer sum: any order gives the same count)
    const int n = __syncthreads_count(acc);
    if (threadIdx.x == 0 && threadIdx.y == 0 && n) atomicAdd(accepted, static_cast<unsigned long long>(n));
}

// sum of the spins (per-block partials summed in block order by the last block)
__global__ void __launch_bounds__(256) k_mc_magnetisation(const double* __restrict__ m, int64_t N, double* partials,
                                                          unsigned int* counter, double* out, int nblocks) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (i < N) {
        v[0] = m[i];
        v[1] = m[N + i];
        v[2] = m[2 * N + i];
    }
    grid_reduce<3>(v, partials, counter, out, nblocks);
}

// The colouring with the fewest colours (at least 2) in which no stencil offset
// joins two sites of one colour: out = {q, b, c, 1} for the linear colour
// (x + b y + c z) mod q, q <= 16, or {cx, cy, cz, 0} for the product colour,
// counts <= 4.  A periodic direction must map its wrapped images to the same
// colour (q divides L0, b L1 and c L2; cx, cy, cz divide the sizes).
bool mc_colouring(const StencilParams& sp, int out[4]) {
    int best = 1 << 30;
    for (int q = 2; q <= 16 && q < best; ++q)
        for (int c = 0; c < q && q < best; ++c)
            for (int b = 0; b < q && q < best; ++b) {
                bool ok = !(sp.periodic[0] && sp.L[0] % q) && !(sp.periodic[1] && (b * sp.L[1]) % q) &&
                          !(sp.periodic[2] && (c * sp.L[2]) % q);
                for (int k = 0; k < sp.n_off && ok; ++k)
                    ok = (((sp.off[k][0] + b * sp.off[k][1] + c * sp.off[k][2]) % q) + q) % q != 0;
                if (ok) {
                    best = q;
                    out[0] = q;
                    out[1] = b;
                    out[2] = c;
                    out[3] = 1;
                }
            }
    for (int cz = 1; cz <= 4; ++cz)
        for (int cy = 1; cy <= 4; ++cy)
            for (int cx = 1; cx <= 4; ++cx) {
                const int cc[3] = {cx, cy, cz};
                bool ok = cx * cy * cz < best && cx * cy * cz > 1;
                for (int d = 0; d < 3 && ok; ++d)
                    if (sp.periodic[d] && sp.L[d] % cc[d] != 0) ok = false;
                for (int k = 0; k < sp.n_off && ok; ++k) {
                    bool differs = false;
                    for (int d = 0; d < 3; ++d) differs = differs || (((sp.off[k][d] % cc[d]) + cc[d]) % cc[d]) != 0;
                    if (!differs) ok = false;
                }
                if (ok) {
                    best = cx * cy * cz;
                    out[0] = cx;
                    out[1] = cy;
                    out[2] = cz;
                    out[3] = 0;
                }
            }
    return best < (1 << 30);
}

}  // namespace
}  // namespace mj

using namespace mj;

extern "C" {

mj_status mj_mc_sweeps(mj_plan* plan, double* m, mj_mc_params* p, int32_t nsweeps, double* E_dev, double* M_dev,
                       int64_t* accepted, int32_t* colors, void* stream) {
    if (!plan || !m || !p || nsweeps < 0) return set_error(MJ_ERR_ARG, "bad Monte Carlo arguments");
    if (!plan->is_stencil || plan->dip_on)
        return set_error(MJ_ERR_UNSUPPORTED, "Monte Carlo sweeps need a single-atom stencil plan, no dipolar term");
    if (p->proposal < MJ_MC_CONE || p->proposal > MJ_MC_OVERRELAX) return set_error(MJ_ERR_ARG, "unknown proposal");
    if (!(p->temperature >= 0.0) || !(p->cone > 0.0)) return set_error(MJ_ERR_ARG, "temperature >= 0 and cone > 0");
    int col[4] = {0, 0, 0, 0};
    if (!mc_colouring(plan->sp, col))
        return set_error(MJ_ERR_UNSUPPORTED, "no linear colouring of at most 16 colours and no product colouring of "
                                             "at most 4 x 4 x 4 fits the stencil and the periodic sizes");
    if (colors)
        for (int d = 0; d < 4; ++d) colors[d] = col[d];
    // the colour classes in launch order
    std::vector<McClass> classes;
    if (col[3] == 1) {
        for (int k = 0; k < col[0]; ++k) classes.push_back({col[0], 1, 1, col[1], col[2], k, 0, 0});
    } else {
        for (int rz = 0; rz < col[2]; ++rz)
            for (int ry = 0; ry < col[1]; ++ry)
                for (int rx = 0; rx < col[0]; ++rx) classes.push_back({col[0], col[1], col[2], 0, 0, rx, ry, rz});
    }
    cudaSetDevice(plan->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t N = plan->N;
    const int nbm = static_cast<int>((N + 255) / 256);
    // the call's scratch: accepted count, ticket counter, magnetisation partials
    struct Scratch {
        unsigned long long acc;
        unsigned int counter[2];
    };
    Scratch* d_scr = nullptr;
    double* d_part = nullptr;
    mj_status st = cuda_status(cudaMalloc(&d_scr, sizeof(Scratch)), "MC scratch");
    if (st == MJ_OK && M_dev) st = cuda_status(cudaMalloc(&d_part, sizeof(double) * 3 * nbm), "MC scratch");
    if (st != MJ_OK) {
        cudaFree(d_scr);
        return st;
    }
    cudaMemsetAsync(d_scr, 0, sizeof(Scratch), s);
    McCoef C;
    std::memset(&C, 0, sizeof(C));
    C.kT = p->temperature * kKB;
    C.proposal = p->proposal;
    C.stream = p->stream_id;
    uint32_t k0 = static_cast<uint32_t>(p->seed), k1 = static_cast<uint32_t>(p->seed >> 32);
    for (int r = 0; r < 10; ++r) {  // Philox4x32 key schedule (Weyl increments)
        C.keys[2 * r] = k0;
        C.keys[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    const McClass& K0 = classes[0];
    const int sub[3] = {(plan->sp.L[0] + K0.qx - 1) / K0.qx, (plan->sp.L[1] + K0.sy - 1) / K0.sy,
                        (plan->sp.L[2] + K0.sz - 1) / K0.sz};
    const dim3 grid((sub[0] + 31) / 32, (sub[1] + 7) / 8, sub[2]), blk(32, 8);
    // the cone rule of sample_sphere (track_value.f90 cone_update: +-1e-4 per move
    // toward an acceptance rate of 0.5, cone in [0.01, pi]), applied once per
    // sweep with the sweep's number of moves and the running rate
    const bool adapt = p->adapt_cone && p->proposal == MJ_MC_CONE;
    int64_t total = 0;
    unsigned long long h_acc = 0;
    auto drain = [&]() -> mj_status {  // accepted moves since the last drain
        mj_status e = cuda_status(cudaMemcpyAsync(&h_acc, &d_scr->acc, sizeof(h_acc), cudaMemcpyDeviceToHost, s),
                                  "MC counters");
        if (e == MJ_OK) e = cuda_status(cudaStreamSynchronize(s), "MC sweeps");
        if (e == MJ_OK) e = cuda_status(cudaMemsetAsync(&d_scr->acc, 0, sizeof(h_acc), s), "MC counters");
        total += static_cast<int64_t>(h_acc);
        p->accepted_total += static_cast<int64_t>(h_acc);
        return e;
    };
    for (int32_t k = 0; k < nsweeps && st == MJ_OK; ++k) {
        C.sweep = p->sweep0 + static_cast<uint32_t>(k);
        C.cos_cone = std::cos(p->cone);
        for (const McClass& K : classes) k_mc_color<<<grid, blk, 0, s>>>(plan->sp, plan->d_bmap, m, C, K, &d_scr->acc);
        if ((st = cuda_status(cudaGetLastError(), "k_mc_color")) != MJ_OK) break;
        if (E_dev && (st = launch_energy(plan, m, E_dev + k, s)) != MJ_OK) break;
        if (M_dev) {
            k_mc_magnetisation<<<nbm, 256, 0, s>>>(m, N, d_part, d_scr->counter, M_dev + 3 * k, nbm);
            if ((st = cuda_status(cudaGetLastError(), "k_mc_magnetisation")) != MJ_OK) break;
        }
        p->proposed_total += N;
        if (adapt) {
            if ((st = drain()) != MJ_OK) break;
            const double rate = static_cast<double>(p->accepted_total) / static_cast<double>(p->proposed_total);
            const double step = 1e-4 * static_cast<double>(N);
            if (rate > 0.5 && p->cone < kPi) p->cone = std::min(kPi, p->cone + step);
            else if (rate < 0.5 && p->cone > 0.01) p->cone = std::max(0.01, p->cone - step);
        }
    }
    if (st == MJ_OK && !adapt) st = drain();
    if (accepted) *accepted = total;
    if (st == MJ_OK) p->sweep0 += static_cast<uint32_t>(nsweeps);
    cudaFree(d_part);
    cudaFree(d_scr);
    return st;
}

}  // extern "C"
