// Metropolis Monte Carlo on the device (Metropolis-MC/MCstep.f90).
//
// The reference makes single-spin moves at random sites (choose_spin.f90).
// Here a sweep moves every site once, colour by colour with a colouring in
// which no coupling joins two sites of one colour, so the moves of a colour are
// independent and run in parallel: the same single-spin moves and acceptance
// rule (mj_mc.cuh) in another site order.  Two families of colourings are
// searched and the one with fewer colours kept: linear, colour (x + b y + c z)
// mod q (2 colours for square and cubic nearest neighbours, 3 for triangular),
// and product, colour (x mod cx, y mod cy, z mod cz); a periodic size must keep
// the colour of its wrapped images.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mj_device.cuh"
#include "mj_internal.hpp"
#include "mj_mc.cuh"

namespace mj {
namespace {

struct McCoef {
    double kT;          // eV
    double inv_kT;      // 1/kT (0 at T = 0)
    double cos_cone;
    const double* tab;  // sin/cos tables (the plan's thermal-draw tables)
    double* track;      // tracked totals: per-block partials [4][track_n] of (dE, dm) of accepted moves, or null
    int track_n;        // partials per component (colours x blocks of a sweep)
    int track_off;      // the first partial of this colour's blocks
    int proposal;       // MJ_MC_*
    uint32_t keys[20];  // Philox round keys of the seed
    uint32_t sweep;
    uint32_t stream;
};

// S: the plan's compile-time stencil shape, void for runtime offsets
template <class S>
__global__ void __launch_bounds__(32 * kMcBY, 8) k_mc_color(const __grid_constant__ StencilParams P, const double* __restrict__ bmap,
                                                  double* m, const McCoef C, const McClass K,
                                                  unsigned long long* accepted) {
    const int y = K.ry + K.sy * static_cast<int>(blockIdx.y * kMcBY + threadIdx.y);
    const int z = K.rz + K.sz * static_cast<int>(blockIdx.z);
    const int x = mc_class_x(K, y, z, static_cast<int>(blockIdx.x * 32 + threadIdx.x));
    bool acc = false;
    double dE = 0.0;
    double3 dm = make_double3(0.0, 0.0, 0.0);
    if (x < P.L[0] && y < P.L[1] && z < P.L[2]) {
        const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
        const int64_t i = x + static_cast<int64_t>(P.L[0]) * (y + static_cast<int64_t>(P.L[1]) * z);
        const double3 s = ld3(m, i, N);
        const double3 Pf = pair_field<S>(P, m, N, P.L[0], P.L[1], P.L[2], x, y, z);
        double3 sn;
        acc = mc_move(P, C.keys, C.tab, C.proposal, C.kT, C.inv_kT, C.cos_cone, static_cast<uint32_t>(i), C.sweep,
                      C.stream, s, Pf, zeeman(P, bmap, i, N), sn, dE);
        if (acc) {
            st3(m, i, N, sn);
            dm = make_double3(sn.x - s.x, sn.y - s.y, sn.z - s.z);
        }
    }
    if (C.track) {  // the block's share of the change of the totals (track_val, MCstep.f90:60-68)
        double v[4] = {acc ? dE : 0.0, dm.x, dm.y, dm.z};
        const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        block_partials<4>(v, C.track, C.track_n, C.track_off + bid);
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

// the totals after a sweep: run = (E, Mx, My, Mz) plus the sweep's partials,
// summed in a fixed order; copied to E_out / M_out when given
__global__ void __launch_bounds__(256) k_mc_track(const double* partials, int n, double* run, double* E_out,
                                                  double* M_out) {
    __shared__ double sum[4];
    ordered_sum<4>(partials, n, sum);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; ++q) run[q] += sum[q];
        if (E_out) *E_out = run[0];
        if (M_out)
            for (int q = 0; q < 3; ++q) M_out[q] = run[1 + q];
    }
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
    if (!mc_colouring(plan->sp, plan->sp.L, 1, col))
        return set_error(MJ_ERR_UNSUPPORTED, "no linear or product colouring fits the stencil and the periodic "
                                             "sizes");
    if (colors)
        for (int d = 0; d < 4; ++d) colors[d] = col[d];
    const std::vector<McClass> classes = mc_classes(col);
    cudaSetDevice(plan->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t N = plan->N;
    const int nbm = static_cast<int>((N + 255) / 256);
    const McClass& K0 = classes[0];
    const int sub[3] = {(plan->sp.L[0] + K0.qx - 1) / K0.qx, (plan->sp.L[1] + K0.sy - 1) / K0.sy,
                        (plan->sp.L[2] + K0.sz - 1) / K0.sz};
    const dim3 grid((sub[0] + 31) / 32, (sub[1] + kMcBY - 1) / kMcBY, sub[2]), blk(32, kMcBY);
    const int nbc = static_cast<int>(grid.x * grid.y * grid.z);  // blocks of one colour pass
    const int ncol = static_cast<int>(classes.size());
    const bool track = p->track_totals && (E_dev || M_dev);
    // the call's scratch: accepted count, ticket counter, running totals (E, M);
    // magnetisation partials; the tracked totals' per-block partials
    struct Scratch {
        unsigned long long acc;
        unsigned int counter[2];
        double run[4];
    };
    Scratch* d_scr = nullptr;
    double* d_part = nullptr;
    double* d_track = nullptr;
    mj_status st = cuda_status(cudaMalloc(&d_scr, sizeof(Scratch)), "MC scratch");
    if (st == MJ_OK && (M_dev || track)) st = cuda_status(cudaMalloc(&d_part, sizeof(double) * 3 * nbm), "MC scratch");
    if (st == MJ_OK && track)
        st = cuda_status(cudaMalloc(&d_track, sizeof(double) * 4 * static_cast<size_t>(ncol) * nbc), "MC scratch");
    if (st != MJ_OK) {
        cudaFree(d_part);
        cudaFree(d_scr);
        return st;
    }
    cudaMemsetAsync(d_scr, 0, sizeof(Scratch), s);
    if (track) {  // the totals at the start of the call
        if ((st = launch_energy(plan, m, &d_scr->run[0], s)) == MJ_OK) {
            k_mc_magnetisation<<<nbm, 256, 0, s>>>(m, N, d_part, d_scr->counter, &d_scr->run[1], nbm);
            st = cuda_status(cudaGetLastError(), "k_mc_magnetisation");
        }
        if (st != MJ_OK) {
            cudaFree(d_track);
            cudaFree(d_part);
            cudaFree(d_scr);
            return st;
        }
    }
    McCoef C;
    std::memset(&C, 0, sizeof(C));
    C.kT = p->temperature * kKB;
    C.inv_kT = C.kT > 0.0 ? 1.0 / C.kT : 0.0;
    C.tab = plan->d_noise_tab;
    C.proposal = p->proposal;
    C.stream = p->stream_id;
    mc_keys(p->seed, C.keys);
    C.track = d_track;
    C.track_n = ncol * nbc;
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
        for (int ci = 0; ci < ncol; ++ci) {
            const McClass& K = classes[ci];
            C.track_off = ci * nbc;
            switch (plan->sp.shape) {
                case kShapeSquareNN:
                    k_mc_color<ShapeSquareNN><<<grid, blk, 0, s>>>(plan->sp, plan->d_bmap, m, C, K, &d_scr->acc);
                    break;
                case kShapeSquare2:
                    k_mc_color<ShapeSquare2><<<grid, blk, 0, s>>>(plan->sp, plan->d_bmap, m, C, K, &d_scr->acc);
                    break;
                case kShapeTriNN:
                    k_mc_color<ShapeTriNN><<<grid, blk, 0, s>>>(plan->sp, plan->d_bmap, m, C, K, &d_scr->acc);
                    break;
                case kShapeTri3:
                    k_mc_color<ShapeTri3><<<grid, blk, 0, s>>>(plan->sp, plan->d_bmap, m, C, K, &d_scr->acc);
                    break;
                default:
                    k_mc_color<void><<<grid, blk, 0, s>>>(plan->sp, plan->d_bmap, m, C, K, &d_scr->acc);
            }
        }
        if ((st = cuda_status(cudaGetLastError(), "k_mc_color")) != MJ_OK) break;
        if (track) {
            k_mc_track<<<1, 256, 0, s>>>(d_track, ncol * nbc, d_scr->run, E_dev ? E_dev + k : nullptr,
                                         M_dev ? M_dev + 3 * k : nullptr);
            if ((st = cuda_status(cudaGetLastError(), "k_mc_track")) != MJ_OK) break;
        } else if (E_dev && (st = launch_energy(plan, m, E_dev + k, s)) != MJ_OK) {
            break;
        }
        if (M_dev && !track) {
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
    cudaFree(d_track);
    cudaFree(d_part);
    cudaFree(d_scr);
    return st;
}

}  // extern "C"
