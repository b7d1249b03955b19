// Reverse mode of the SIB trajectory: gradients of a loss of the final spins
// with respect to the initial spins, the coupling-term values (exchange, DMI,
// anisotropy, in the order of the Hamiltonian description) and the per-site
// applied field.  The reference has no derivative code; the forward map is the
// SIB step of the dynamics (Mentink et al. 2010, the stage loop of
// dynamics/spindynamics.f90:282-313) with the effective field of
// Hamiltonian_type/hamiltonian_collection.f90:433-454.
//
// Forward step n (H = W m + zc b + thermal draw, W the symmetric stencil
// operator of all real-space terms: W_{-o}^T = W_o):
//   H1 = H(m_n);  y1 = S(m_n, m_n, H1);  mb = (m_n + y1)/2
//   H2 = H(mb);   m_{n+1} = S(m_n, mb, H2)
// with S the closed-form Cayley solve.  Backward step n, g = dL/dm_{n+1}:
//   (gm2, gp2, gH2) = S^T(m_n, mb, H2; g)
//   gmb = gp2 + W gH2                       (W^T = W)
//   (gm1, gp1, gH1) = S^T(m_n, m_n, H1; gmb/2)
//   dL/dm_n = gm2 + gmb/2 + gm1 + gp1 + W gH1
//   dL/dv_t += gH2 . W_t mb + gH1 . W_t m_n,   dL/db_i += zc (gH1_i + gH2_i)
// Kernels per backward step: k_adj_ca (the W gH1 of step n+1 fused with the
// stage-2 transpose of step n) and k_adj_b (W gH2, stage-1 transpose), each as
// a tiled kernel over a compile-time stencil shape (both stencil inputs staged
// in shared memory, every offset unrolled) or, for other lattices, a generic
// one-site-per-thread kernel.  The trajectory is checkpointed every
// `checkpoint_every` steps; each segment is recomputed (m_n and mb stored)
// with the plan's own SIB kernels before its backward sweep.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "mj_device.cuh"
#include "mj_internal.hpp"
#include "mj_stencil.cuh"
#include "mj_tiled_impl.cuh"

namespace mj {
namespace {

constexpr int kMaxTerms = 8;   // differentiable coupling terms of a plan
constexpr int kABX = 32, kABY = 8;

__device__ __forceinline__ bool adj_site(const StencilParams& P, int64_t& i, int& x, int& y, int& z) {
    x = blockIdx.x * kABX + threadIdx.x;
    y = blockIdx.y * kABY + threadIdx.y;
    z = blockIdx.z;
    const bool a = x < P.L[0] && y < P.L[1];
    i = a ? x + static_cast<int64_t>(P.L[0]) * (y + static_cast<int64_t>(P.L[1]) * z) : 0;
    return a;
}

// Which unit tensors are nonzero / isotropic: bit k of nz[t] (iso[t]) for offset
// k of term t, bit n_off for the on-site tensor.
struct TermMasks {
    unsigned long long nz[kMaxTerms];
    unsigned long long iso[kMaxTerms];
    unsigned long long any;  // OR of nz
    int nterm;
};

// acc[t] += g . (W_t v)_i for every term t (unit tensors [nterm][n_off+1][9])
__device__ __forceinline__ void term_grads(const StencilParams& P, const double* __restrict__ unit, const TermMasks& M,
                                           const double* __restrict__ v, int64_t N, int x, int y, int z, double3 v0,
                                           double3 g, double* acc) {
    const int stride = (P.n_off + 1) * 9;
    for (int k = 0; k <= P.n_off; ++k) {
        if (!((M.any >> k) & 1ull)) continue;
        double3 a;
        if (k < P.n_off) {
            int64_t j;
            if (!neighbour(P, x, y, z, k, j)) continue;
            a = ld3(v, j, N);
        } else {
            a = v0;
        }
        const double ga = dot(g, a);
#pragma unroll
        for (int t = 0; t < kMaxTerms; ++t) {
            if (t < M.nterm && ((M.nz[t] >> k) & 1ull)) {
                const double* U = unit + t * stride + k * 9;
                if ((M.iso[t] >> k) & 1ull) {
                    acc[t] = fma(__ldg(U), ga, acc[t]);
                } else {
                    const double3 u = mat3(U, a, make_double3(0.0, 0.0, 0.0));
                    acc[t] = fma(g.x, u.x, fma(g.y, u.y, fma(g.z, u.z, acc[t])));
                }
            }
        }
    }
}

// Deterministic grid reduction of the first nq of kMaxTerms values (blocks of
// 256 threads): per-block partials, summed in block order by the last block.
__device__ void term_reduce(const double* acc, int nq, double* partials, unsigned int* counter, double* out,
                            int nblocks) {
    __shared__ double wsum[kMaxTerms][8];
    __shared__ bool last;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
    const int lane = tid & 31, wid = tid >> 5;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
#pragma unroll
    for (int q = 0; q < kMaxTerms; ++q) {
        if (q < nq) {
            double e = acc[q];
            for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
            if (lane == 0) wsum[q][wid] = e;
        }
    }
    __syncthreads();
    if (tid == 0) {
        for (int q = 0; q < nq; ++q) {
            double sum = 0.0;
            for (int w = 0; w < nthr / 32; ++w) sum += wsum[q][w];
            partials[static_cast<int64_t>(q) * nblocks + bid] = sum;
        }
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == static_cast<unsigned int>(nblocks - 1));
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int q = 0; q < nq; ++q) {
        double sum = 0.0;
        for (int b = tid; b < nblocks; b += nthr) sum += __ldcg(partials + static_cast<int64_t>(q) * nblocks + b);
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        __syncthreads();
        if (lane == 0) wsum[0][wid] = sum;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < nthr / 32; ++w) t += wsum[0][w];
            out[q] = t;
        }
    }
    if (tid == 0) *counter = 0u;
}

// Transpose of the SIB solve y = S(m, p, H): returns dL/dm, dL/dp, dL/dH given dL/dy.
struct SibGrad {
    double3 gm, gp, gH;
};
__device__ __forceinline__ SibGrad sib_vjp(double3 m, double3 p, double3 H, double alpha, double hc, double3 gy) {
    const double np2 = dot(p, p);
    const bool norm = np2 > 1e-16;
    double3 pn = p;
    double invn = 1.0;
    if (norm) {
        invn = rsqrt(np2);
        pn = scl3(invn, p);
    }
    const double3 pxh = cross(pn, H);
    const double3 h = scl3(hc, make_double3(H.x + alpha * pxh.x, H.y + alpha * pxh.y, H.z + alpha * pxh.z));
    // y = m + c (u + w), u = m x h, w = u x h, c = 2/(1 + h.h)
    const double3 u = cross(m, h);
    const double3 w = cross(u, h);
    const double c = 2.0 / (1.0 + dot(h, h));
    SibGrad r;
    r.gm = gy;
    const double gc = dot(gy, add3(u, w));
    const double3 gw = scl3(c, gy);
    double3 gu = add3(scl3(c, gy), cross(h, gw));  // w = u x h: u gets h x gw
    double3 gh = cross(gw, u);                      //            h gets gw x u
    r.gm = add3(r.gm, cross(h, gu));                // u = m x h: m gets h x gu
    gh = add3(gh, cross(gu, m));                    //            h gets gu x m
    gh = add3(gh, scl3(-gc * c * c, h));            // c = 2/s: dc/dh = -c^2 h
    // h = hc (H + alpha p^ x H)
    const double3 uu = scl3(hc * alpha, gh);
    r.gH = add3(scl3(hc, gh), cross(uu, pn));
    const double3 gpn = cross(H, uu);
    r.gp = norm ? scl3(invn, make_double3(gpn.x - dot(pn, gpn) * pn.x, gpn.y - dot(pn, gpn) * pn.y,
                                          gpn.z - dot(pn, gpn) * pn.z))
                : gpn;
    return r;
}

__device__ __forceinline__ double3 noise(const DynCoef& C, uint32_t step, int64_t i, int64_t N) {
    if (!C.thermal) return make_double3(0.0, 0.0, 0.0);
    return thermal_field(C, step, i, N);
}

struct AdjReduce {
    double* partials;      // [kMaxTerms][nblocks]
    unsigned int* counter;
    double* slot;          // kMaxTerms doubles for this launch
    int nblocks;
};

// ---------------------------------------------------------------------------
// forward passes (explicit buffers): mb = (m_n + S(m_n, m_n, H(m_n)))/2, m_{n+1} = S(m_n, mb, H(mb))
__global__ void __launch_bounds__(256) k_adj_f1(const __grid_constant__ StencilParams P, const DynCoef C, uint32_t step,
                                                const double* __restrict__ bmap, const double* __restrict__ m,
                                                double* __restrict__ mb) {
    int64_t i;
    int x, y, z;
    if (!adj_site(P, i, x, y, z)) return;
    const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
    const double3 m0 = ld3(m, i, N);
    const double3 H = add3(add3(w_apply(P, m, N, x, y, z, m0), zeeman(P, bmap, i, N)), noise(C, step, i, N));
    st3(mb, i, N, sib_solve<true>(m0, m0, H, C.alpha, C.sib_hc));
}

__global__ void __launch_bounds__(256) k_adj_f2(const __grid_constant__ StencilParams P, const DynCoef C, uint32_t step,
                                                const double* __restrict__ bmap, const double* __restrict__ m,
                                                const double* __restrict__ mb, double* __restrict__ mout) {
    int64_t i;
    int x, y, z;
    if (!adj_site(P, i, x, y, z)) return;
    const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
    const double3 b0 = ld3(mb, i, N);
    const double3 H = add3(add3(w_apply(P, mb, N, x, y, z, b0), zeeman(P, bmap, i, N)), noise(C, step, i, N));
    st3(mout, i, N, sib_solve(ld3(m, i, N), b0, H, C.alpha, C.sib_hc));
}

// ---------------------------------------------------------------------------
// backward: g = mpart + W gH1 (the end of step n+1's transpose; gT itself when
// gH1 is null), then, unless mb is null, the stage-2 transpose of step n.
__global__ void __launch_bounds__(256) k_adj_ca(const __grid_constant__ StencilParams P, const DynCoef C, uint32_t step,
                                                const double* __restrict__ bmap, const double* __restrict__ unit,
                                                const TermMasks M, const double* __restrict__ gH1,
                                                const double* __restrict__ mpart, const double* __restrict__ m,
                                                const double* __restrict__ mb, double* __restrict__ g_out,
                                                double* __restrict__ gH2, double* __restrict__ gp2,
                                                double* __restrict__ gm2, AdjReduce R) {
    int64_t i;
    int x, y, z;
    const bool act = adj_site(P, i, x, y, z);
    const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
    double acc[kMaxTerms];
#pragma unroll
    for (int t = 0; t < kMaxTerms; ++t) acc[t] = 0.0;
    if (act) {
        double3 g = ld3(mpart, i, N);
        if (gH1) g = add3(g, w_apply(P, gH1, N, x, y, z, ld3(gH1, i, N)));
        if (!mb) {
            st3(g_out, i, N, g);
        } else {
            const double3 b0 = ld3(mb, i, N);
            const double3 H2 =
                add3(add3(w_apply(P, mb, N, x, y, z, b0), zeeman(P, bmap, i, N)), noise(C, step, i, N));
            const SibGrad s = sib_vjp(ld3(m, i, N), b0, H2, C.alpha, C.sib_hc, g);
            st3(gH2, i, N, s.gH);
            st3(gp2, i, N, s.gp);
            st3(gm2, i, N, s.gm);
            if (M.nterm > 0) term_grads(P, unit, M, mb, N, x, y, z, b0, s.gH, acc);
        }
    }
    if (mb && M.nterm > 0) term_reduce(acc, M.nterm, R.partials, R.counter, R.slot, R.nblocks);
}

// backward, stage 1 of step n: gmb = gp2 + W gH2, stage-1 transpose, field gradient
__global__ void __launch_bounds__(256) k_adj_b(const __grid_constant__ StencilParams P, const DynCoef C, uint32_t step,
                                               const double* __restrict__ bmap, const double* __restrict__ unit,
                                               const TermMasks M, const double* __restrict__ gH2,
                                               const double* __restrict__ gp2, const double* __restrict__ gm2,
                                               const double* __restrict__ m, double* __restrict__ gH1,
                                               double* __restrict__ mpart, double* __restrict__ gb, AdjReduce R) {
    int64_t i;
    int x, y, z;
    const bool act = adj_site(P, i, x, y, z);
    const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
    double acc[kMaxTerms];
#pragma unroll
    for (int t = 0; t < kMaxTerms; ++t) acc[t] = 0.0;
    if (act) {
        const double3 h2 = ld3(gH2, i, N);
        const double3 gmb = add3(ld3(gp2, i, N), w_apply(P, gH2, N, x, y, z, h2));
        const double3 gy1 = scl3(0.5, gmb);
        const double3 m0 = ld3(m, i, N);
        const double3 H1 = add3(add3(w_apply(P, m, N, x, y, z, m0), zeeman(P, bmap, i, N)), noise(C, step, i, N));
        const SibGrad s = sib_vjp(m0, m0, H1, C.alpha, C.sib_hc, gy1);
        st3(gH1, i, N, s.gH);
        st3(mpart, i, N, add3(add3(ld3(gm2, i, N), gy1), add3(s.gm, s.gp)));
        if (gb && P.zee_on) {
            const double3 prev = ld3(gb, i, N);
            st3(gb, i, N, add3(prev, scl3(P.zc, add3(s.gH, h2))));
        }
        if (M.nterm > 0) term_grads(P, unit, M, m, N, x, y, z, m0, s.gH, acc);
    }
    if (M.nterm > 0) term_reduce(acc, M.nterm, R.partials, R.counter, R.slot, R.nblocks);
}

// sum of the per-launch term gradients in launch order
__global__ void k_adj_sum(const double* __restrict__ slots, int nslot, int nterm, double* __restrict__ out) {
    const int t = threadIdx.x;
    if (t >= nterm) return;
    double s = 0.0;
    for (int k = 0; k < nslot; ++k) s += slots[static_cast<int64_t>(k) * kMaxTerms + t];
    out[t] = s;
}

// VJP of the field: g_m = W v, g_terms[t] = v . W_t m, g_b = zc v (per site)
__global__ void __launch_bounds__(256) k_field_vjp(const __grid_constant__ StencilParams P,
                                                   const double* __restrict__ unit, const TermMasks M,
                                                   const double* __restrict__ m, const double* __restrict__ v,
                                                   double* __restrict__ gm, double* __restrict__ gb, AdjReduce R) {
    int64_t i;
    int x, y, z;
    const bool act = adj_site(P, i, x, y, z);
    const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
    double acc[kMaxTerms];
#pragma unroll
    for (int t = 0; t < kMaxTerms; ++t) acc[t] = 0.0;
    if (act) {
        const double3 v0 = ld3(v, i, N);
        if (gm) st3(gm, i, N, w_apply(P, v, N, x, y, z, v0));
        if (gb) st3(gb, i, N, P.zee_on ? scl3(P.zc, v0) : make_double3(0.0, 0.0, 0.0));
        if (M.nterm > 0) term_grads(P, unit, M, m, N, x, y, z, ld3(m, i, N), v0, acc);
    }
    if (M.nterm > 0 && R.slot) term_reduce(acc, M.nterm, R.partials, R.counter, R.slot, R.nblocks);
}


// ---------------------------------------------------------------------------
// Tiled backward kernels for the compile-time shapes (mj_shapes.hpp).  A block
// of 32 x BYT threads owns a 32 x BYT*RY tile; the two stencil inputs of the
// kernel are staged with their halo in shared memory (TileGeom layout), the
// unit tensors of the terms follow them.  W v reuses the forward column walk
// (all_columns); the per-term stencils W_t v walk the same tile with the unit
// tensors read from shared memory, skipping zero tensors and taking one load
// for isotropic ones.
template <class S, int RY, int DX, int YY, int... Kk>
__device__ __forceinline__ void unit_row(const double* U, unsigned long long nz, unsigned long long iso, double vx,
                                         double vy, double vz, double* bx, double* by, double* bz,
                                         std::integer_sequence<int, Kk...>) {
    (
        [&] {
            constexpr int k = Kk;
            if constexpr (S::DX[k] == DX) {
                constexpr int r = YY - S::DY[k];
                if constexpr (r >= 0 && r < RY) {
                    if ((nz >> k) & 1ull) {
                        const double* W = U + 9 * k;
                        if ((iso >> k) & 1ull) {
                            const double w = W[0];
                            bx[r] = fma(w, vx, bx[r]);
                            by[r] = fma(w, vy, by[r]);
                            bz[r] = fma(w, vz, bz[r]);
                        } else {
                            bx[r] = fma(W[0], vx, fma(W[1], vy, fma(W[2], vz, bx[r])));
                            by[r] = fma(W[3], vx, fma(W[4], vy, fma(W[5], vz, by[r])));
                            bz[r] = fma(W[6], vx, fma(W[7], vy, fma(W[8], vz, bz[r])));
                        }
                    }
                }
            }
        }(),
        ...);
}

template <class S, int BYT, int RY, int DX, int... Y>
__device__ __forceinline__ void unit_column(const double* U, unsigned long long nz, unsigned long long iso,
                                            const double* sm, int base, double* bx, double* by, double* bz,
                                            std::integer_sequence<int, Y...>) {
    using G = TileGeom<S, BYT, RY>;
    constexpr int ylo = shape_col_ymin<S>(DX);
    (
        [&] {
            constexpr int yy = ylo + Y;
            const int s = base + (yy + G::R) * G::PX + DX + G::RX;
            unit_row<S, RY, DX, yy>(U, nz, iso, sm[s], sm[G::NS + s], sm[2 * G::NS + s], bx, by, bz,
                                    std::make_integer_sequence<int, S::K>{});
        }(),
        ...);
}

template <class S, int BYT, int RY, int... Cc>
__device__ __forceinline__ void unit_columns(const double* U, unsigned long long nz, unsigned long long iso,
                                             const double* sm, int base, double* bx, double* by, double* bz,
                                             std::integer_sequence<int, Cc...>) {
    (
        [&] {
            constexpr int dx = Cc - S::R;
            constexpr int ylo = shape_col_ymin<S>(dx), yhi = shape_col_ymax<S>(dx);
            if constexpr (ylo <= yhi) {
                unit_column<S, BYT, RY, dx>(U, nz, iso, sm, base, bx, by, bz,
                                            std::make_integer_sequence<int, RY + yhi - ylo>{});
            }
        }(),
        ...);
}

// acc[t] += g_r . (W_t v)_r over the thread's RY sites, v staged in `tile`
template <class S, int BYT, int RY>
__device__ __forceinline__ void tiled_term_grads(const double* Us, const TermMasks& M, const double* tile, int base,
                                                 const double3* g, const bool* act, double* acc) {
    using G = TileGeom<S, BYT, RY>;
#pragma unroll
    for (int t = 0; t < kMaxTerms; ++t) {
        if (t < M.nterm) {
            const double* U = Us + t * (S::K + 1) * 9;
            double ux[RY], uy[RY], uz[RY];
#pragma unroll
            for (int r = 0; r < RY; ++r) ux[r] = uy[r] = uz[r] = 0.0;
            unit_columns<S, BYT, RY>(U, M.nz[t], M.iso[t], tile, base, ux, uy, uz,
                                     std::make_integer_sequence<int, 2 * S::R + 1>{});
            const bool onsite = (M.nz[t] >> S::K) & 1ull;
            const double* U0 = U + 9 * S::K;
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                if (!act[r]) continue;
                double3 u = make_double3(ux[r], uy[r], uz[r]);
                if (onsite) {
                    const int c = base + (r + G::R) * G::PX + G::RX;
                    u = mat3(U0, make_double3(tile[c], tile[G::NS + c], tile[2 * G::NS + c]), u);
                }
                acc[t] = fma(g[r].x, u.x, fma(g[r].y, u.y, fma(g[r].z, u.z, acc[t])));
            }
        }
    }
}

// W v at the thread's RY sites (main stencil + on-site tensor), v staged in `tile`
template <class S, int BYT, int RY>
__device__ __forceinline__ void tiled_apply(const StencilParams& P, const double* tile, int base, double3* out) {
    using G = TileGeom<S, BYT, RY>;
    double bx[RY], by[RY], bz[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) bx[r] = by[r] = bz[r] = 0.0;
    all_columns<S, BYT, RY>(P, tile, base, bx, by, bz, std::make_integer_sequence<int, 2 * S::R + 1>{});
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        out[r] = make_double3(bx[r], by[r], bz[r]);
        if (P.has_onsite) {
            const int c = base + (r + G::R) * G::PX + G::RX;
            out[r] = mat3(P.W0, make_double3(tile[c], tile[G::NS + c], tile[2 * G::NS + c]), out[r]);
        }
    }
}

template <class S, int BYT, int RY>
__device__ __forceinline__ void stage_units(const double* __restrict__ unit, const TermMasks& M, double* Us) {
    const int tid = threadIdx.x + 32 * threadIdx.y;
    const int nu = M.nterm * (S::K + 1) * 9;
    for (int q = tid; q < nu; q += 32 * BYT) Us[q] = __ldg(unit + q);
}

template <class S, int BYT, int RY>
__global__ void __launch_bounds__(32 * BYT) k_tadj_ca(const __grid_constant__ StencilParams P, const DynCoef C,
                                                      uint32_t step, const double* __restrict__ bmap,
                                                      const double* __restrict__ unit, const TermMasks M,
                                                      const double* __restrict__ gH1, const double* __restrict__ mpart,
                                                      const double* __restrict__ m, const double* __restrict__ mb,
                                                      double* __restrict__ g_out, double* __restrict__ gH2,
                                                      double* __restrict__ gp2, double* __restrict__ gm2,
                                                      AdjReduce R) {
    using G = TileGeom<S, BYT, RY>;
    extern __shared__ __align__(128) double smem_a[];
    double* tA = smem_a;               // gH1
    double* tB = smem_a + 3 * G::NS;   // mb
    double* Us = smem_a + 6 * G::NS;   // unit tensors
    const int x0 = blockIdx.x * G::TX, y0 = blockIdx.y * G::TY;
    const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1];
    if (gH1) load_tile<S, BYT, RY>(P, gH1, x0, y0, 0, tA);
    if (mb) load_tile<S, BYT, RY>(P, mb, x0, y0, 0, tB);
    if (mb) stage_units<S, BYT, RY>(unit, M, Us);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int base = (ty * RY) * G::PX + tx;
    const int x = x0 + tx;
    double3 g[RY], wg[RY];
    bool act[RY];
    int64_t idx[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int y = y0 + ty * RY + r;
        act[r] = x < P.L[0] && y < P.L[1];
        idx[r] = act[r] ? x + static_cast<int64_t>(P.L[0]) * y : 0;
        g[r] = act[r] ? ld3(mpart, idx[r], N) : make_double3(0.0, 0.0, 0.0);
    }
    if (gH1) {
        tiled_apply<S, BYT, RY>(P, tA, base, wg);
#pragma unroll
        for (int r = 0; r < RY; ++r) g[r] = add3(g[r], wg[r]);
    }
    double acc[kMaxTerms];
#pragma unroll
    for (int t = 0; t < kMaxTerms; ++t) acc[t] = 0.0;
    if (!mb) {
#pragma unroll
        for (int r = 0; r < RY; ++r)
            if (act[r]) st3(g_out, idx[r], N, g[r]);
        return;
    }
    double3 H[RY];
    tiled_apply<S, BYT, RY>(P, tB, base, H);
    double3 gh[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        gh[r] = make_double3(0.0, 0.0, 0.0);
        if (!act[r]) continue;
        const int c = base + (r + G::R) * G::PX + G::RX;
        const double3 b0 = make_double3(tB[c], tB[G::NS + c], tB[2 * G::NS + c]);
        const double3 H2 = add3(add3(H[r], zeeman(P, bmap, idx[r], N)), noise(C, step, idx[r], N));
        const SibGrad sg = sib_vjp(ld3(m, idx[r], N), b0, H2, C.alpha, C.sib_hc, g[r]);
        st3(gH2, idx[r], N, sg.gH);
        st3(gp2, idx[r], N, sg.gp);
        st3(gm2, idx[r], N, sg.gm);
        gh[r] = sg.gH;
    }
    if (M.nterm > 0) {
        tiled_term_grads<S, BYT, RY>(Us, M, tB, base, gh, act, acc);
        term_reduce(acc, M.nterm, R.partials, R.counter, R.slot, R.nblocks);
    }
}

template <class S, int BYT, int RY>
__global__ void __launch_bounds__(32 * BYT) k_tadj_b(const __grid_constant__ StencilParams P, const DynCoef C,
                                                     uint32_t step, const double* __restrict__ bmap,
                                                     const double* __restrict__ unit, const TermMasks M,
                                                     const double* __restrict__ gH2, const double* __restrict__ gp2,
                                                     const double* __restrict__ gm2, const double* __restrict__ m,
                                                     double* __restrict__ gH1, double* __restrict__ mpart,
                                                     double* __restrict__ gb, AdjReduce R) {
    using G = TileGeom<S, BYT, RY>;
    extern __shared__ __align__(128) double smem_b[];
    double* tA = smem_b;               // gH2
    double* tB = smem_b + 3 * G::NS;   // m_n
    double* Us = smem_b + 6 * G::NS;
    const int x0 = blockIdx.x * G::TX, y0 = blockIdx.y * G::TY;
    const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1];
    load_tile<S, BYT, RY>(P, gH2, x0, y0, 0, tA);
    load_tile<S, BYT, RY>(P, m, x0, y0, 0, tB);
    stage_units<S, BYT, RY>(unit, M, Us);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int base = (ty * RY) * G::PX + tx;
    const int x = x0 + tx;
    double3 wg[RY], H[RY], gh[RY];
    bool act[RY];
    int64_t idx[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int y = y0 + ty * RY + r;
        act[r] = x < P.L[0] && y < P.L[1];
        idx[r] = act[r] ? x + static_cast<int64_t>(P.L[0]) * y : 0;
    }
    tiled_apply<S, BYT, RY>(P, tA, base, wg);
    tiled_apply<S, BYT, RY>(P, tB, base, H);
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        gh[r] = make_double3(0.0, 0.0, 0.0);
        if (!act[r]) continue;
        const int c = base + (r + G::R) * G::PX + G::RX;
        const double3 h2 = make_double3(tA[c], tA[G::NS + c], tA[2 * G::NS + c]);
        const double3 m0 = make_double3(tB[c], tB[G::NS + c], tB[2 * G::NS + c]);
        const double3 gmb = add3(ld3(gp2, idx[r], N), wg[r]);
        const double3 gy1 = scl3(0.5, gmb);
        const double3 H1 = add3(add3(H[r], zeeman(P, bmap, idx[r], N)), noise(C, step, idx[r], N));
        const SibGrad sg = sib_vjp(m0, m0, H1, C.alpha, C.sib_hc, gy1);
        st3(gH1, idx[r], N, sg.gH);
        st3(mpart, idx[r], N, add3(add3(ld3(gm2, idx[r], N), gy1), add3(sg.gm, sg.gp)));
        if (gb && P.zee_on) st3(gb, idx[r], N, add3(ld3(gb, idx[r], N), scl3(P.zc, add3(sg.gH, h2))));
        gh[r] = sg.gH;
    }
    if (M.nterm > 0) {
        double acc[kMaxTerms];
#pragma unroll
        for (int t = 0; t < kMaxTerms; ++t) acc[t] = 0.0;
        tiled_term_grads<S, BYT, RY>(Us, M, tB, base, gh, act, acc);
        term_reduce(acc, M.nterm, R.partials, R.counter, R.slot, R.nblocks);
    }
}

// tile shape of the tiled backward: 32 x 8 sites, one per thread
constexpr int kTBYT = 8, kTRY = 1;

template <class S>
size_t tadj_smem(int nterm) {
    using G = TileGeom<S, kTBYT, kTRY>;
    return sizeof(double) * (6 * G::NS + static_cast<size_t>(nterm) * (S::K + 1) * 9);
}

template <class S>
dim3 tadj_grid(const StencilParams& P) {
    using G = TileGeom<S, kTBYT, kTRY>;
    return dim3((P.L[0] + G::TX - 1) / G::TX, (P.L[1] + G::TY - 1) / G::TY, 1);
}

struct CaArgs {
    uint32_t step;
    const double *gH1, *mpart, *m, *mb;
    double *g_out, *gH2, *gp2, *gm2;
    AdjReduce R;
};
struct BArgs {
    uint32_t step;
    const double *gH2, *gp2, *gm2, *m;
    double *gH1, *mpart, *gb;
    AdjReduce R;
};

template <class S>
void tadj_launch(const mj_plan* plan, const DynCoef& c, const TermMasks& M, const CaArgs* ca, const BArgs* b,
                 cudaStream_t s) {
    const size_t sm = tadj_smem<S>(M.nterm);
    const dim3 grid = tadj_grid<S>(plan->sp), blk(32, kTBYT);
    if (ca)
        k_tadj_ca<S, kTBYT, kTRY><<<grid, blk, sm, s>>>(plan->sp, c, ca->step, plan->d_bmap, plan->d_unit, M, ca->gH1,
                                                       ca->mpart, ca->m, ca->mb, ca->g_out, ca->gH2, ca->gp2, ca->gm2,
                                                       ca->R);
    if (b)
        k_tadj_b<S, kTBYT, kTRY><<<grid, blk, sm, s>>>(plan->sp, c, b->step, plan->d_bmap, plan->d_unit, M, b->gH2,
                                                      b->gp2, b->gm2, b->m, b->gH1, b->mpart, b->gb, b->R);
}

// the tiled backward kernels of the plan's shape; false when none applies
bool tadj_dispatch(const mj_plan* plan, const DynCoef& c, const TermMasks& M, const CaArgs* ca, const BArgs* b,
                   cudaStream_t s) {
    if (plan->sp.L[2] != 1) return false;
    switch (plan->sp.shape) {
        case kShapeSquareNN: tadj_launch<ShapeSquareNN>(plan, c, M, ca, b, s); return true;
        case kShapeSquare2: tadj_launch<ShapeSquare2>(plan, c, M, ca, b, s); return true;
        case kShapeTriNN: tadj_launch<ShapeTriNN>(plan, c, M, ca, b, s); return true;
        case kShapeTri3: tadj_launch<ShapeTri3>(plan, c, M, ca, b, s); return true;
        default: return false;
    }
}

dim3 adj_grid(const StencilParams& P) {
    return dim3((P.L[0] + kABX - 1) / kABX, (P.L[1] + kABY - 1) / kABY, P.L[2]);
}

int plan_nterm(const mj_plan* p) {
    return static_cast<int>(p->termJ.size() + p->termD.size() + p->termK.size());
}

// nonzero / isotropic masks of the unit tensors (nterm = 0 gives an empty set)
TermMasks term_masks(const mj_plan* p, int nterm) {
    TermMasks M;
    std::memset(&M, 0, sizeof(M));
    M.nterm = nterm;
    const int n_off = p->sp.n_off;
    for (int t = 0; t < nterm; ++t)
        for (int k = 0; k <= n_off; ++k) {
            const double* U = p->unitW.data() + (static_cast<size_t>(t) * (n_off + 1) + k) * 9;
            bool nz = false, iso = U[0] == U[4] && U[0] == U[8];
            for (int q = 0; q < 9; ++q) {
                nz = nz || U[q] != 0.0;
                if (q != 0 && q != 4 && q != 8 && U[q] != 0.0) iso = false;
            }
            if (nz) M.nz[t] |= 1ull << k;
            if (nz && iso) M.iso[t] |= 1ull << k;
            if (nz) M.any |= 1ull << k;
        }
    return M;
}

// per-term unit stencils in the plan's offset order
mj_status ensure_units(mj_plan* p) {
    if (!p->unitW.empty() || plan_nterm(p) == 0) return MJ_OK;
    if (!p->is_stencil) return set_error(MJ_ERR_UNSUPPORTED, "coupling-term gradients need a single-atom stencil plan");
    const int nt = plan_nterm(p);
    const int n_off = p->sp.n_off;
    std::vector<double> U(static_cast<size_t>(nt) * (n_off + 1) * 9, 0.0);
    for (int t = 0; t < nt; ++t) {
        mj_hamiltonian_desc h = p->ham;
        h.nJ = h.nD = h.nK = 0;
        h.J = nullptr;
        h.D = nullptr;
        h.K = nullptr;
        h.zeeman_on = 0;
        h.dip_on = 0;
        h.B_ext[0] = h.B_ext[1] = h.B_ext[2] = 0.0;
        mj_exchange_term ej;
        mj_dmi_term ed;
        mj_aniso_term ek;
        const int nJ = static_cast<int>(p->termJ.size()), nD = static_cast<int>(p->termD.size());
        if (t < nJ) {
            ej = p->termJ[t];
            ej.value = 1.0;
            h.nJ = 1;
            h.J = &ej;
        } else if (t < nJ + nD) {
            ed = p->termD[t - nJ];
            ed.value = 1.0;
            h.nD = 1;
            h.D = &ed;
        } else {
            ek = p->termK[t - nJ - nD];
            ek.value = 1.0;
            h.nK = 1;
            h.K = &ek;
        }
        std::vector<Block> blocks;
        std::vector<double> onsite;
        std::string err;
        if (!build_blocks(p->geom, h, blocks, onsite, err)) return set_error(MJ_ERR_GEOMETRY, err);
        StencilParams u;
        std::memset(&u, 0, sizeof(u));
        if (!stencil_from_blocks(blocks, onsite, u)) return set_error(MJ_ERR_UNSUPPORTED, "term stencil too wide");
        double* Ut = U.data() + static_cast<size_t>(t) * (n_off + 1) * 9;
        for (int k = 0; k < u.n_off; ++k) {
            int j = -1;
            for (int q = 0; q < n_off; ++q)
                if (p->sp.off[q][0] == u.off[k][0] && p->sp.off[q][1] == u.off[k][1] && p->sp.off[q][2] == u.off[k][2])
                    j = q;
            bool nonzero = false;
            for (int q = 0; q < 9; ++q) nonzero = nonzero || u.W[k][q] != 0.0;
            if (j < 0) {
                if (nonzero) return set_error(MJ_ERR_GEOMETRY, "term offset missing from the plan's stencil");
                continue;
            }
            for (int q = 0; q < 9; ++q) Ut[j * 9 + q] = u.W[k][q];
        }
        for (int q = 0; q < 9; ++q) Ut[n_off * 9 + q] = u.W0[q];
    }
    mj_status st = cuda_status(cudaMalloc(&p->d_unit, sizeof(double) * U.size()), "unit stencils");
    if (st != MJ_OK) return st;
    if ((st = cuda_status(cudaMemcpy(p->d_unit, U.data(), sizeof(double) * U.size(), cudaMemcpyHostToDevice),
                          "unit stencils")) != MJ_OK)
        return st;
    p->unitW.swap(U);
    return MJ_OK;
}

}  // namespace
}  // namespace mj

// ---------------------------------------------------------------------------
struct mj_adjoint {
    mj_plan* plan = nullptr;
    int32_t nsteps = 0;
    int32_t every = 1;
    int32_t nseg = 0;
    int64_t N = 0;
    int nblocks = 0;
    bool have_forward = false;
    mj_dyn_params prm{};
    double* d_ckpt = nullptr;   // [nseg + 1][3N]
    double* d_segm = nullptr;   // [every][3N] (slot 0 unused: the checkpoint itself)
    double* d_segb = nullptr;   // [every][3N]
    double* d_work = nullptr;   // [3][3N]: forward ping-pong + midpoint
    double* d_gH1 = nullptr;
    double* d_mpart = nullptr;
    double* d_gH2 = nullptr;
    double* d_gp2 = nullptr;
    double* d_gm2 = nullptr;
    double* d_gin = nullptr;    // the incoming dL/dm_T
    double* d_partials = nullptr;
    unsigned int* d_counter = nullptr;
    double* d_slots = nullptr;  // [2 nsteps][kMaxTerms]
    double* d_g0 = nullptr;     // outputs of the backward sweep (copied to the caller's buffers)
    double* d_gterms = nullptr; // kMaxTerms
    double* d_gb = nullptr;     // 3N
    // the two sweeps as CUDA graphs over the buffers above, cached with their key
    cudaStream_t cap = nullptr;
    cudaGraphExec_t gfwd = nullptr, gbwd = nullptr;
    std::string kfwd, kbwd;
};

namespace mj {
namespace {

void adjoint_free(mj_adjoint* a) {
    if (!a) return;
    if (a->gfwd) cudaGraphExecDestroy(a->gfwd);
    if (a->gbwd) cudaGraphExecDestroy(a->gbwd);
    if (a->cap) cudaStreamDestroy(a->cap);
    cudaFree(a->d_g0);
    cudaFree(a->d_gterms);
    cudaFree(a->d_gb);
    cudaFree(a->d_ckpt);
    cudaFree(a->d_segm);
    cudaFree(a->d_segb);
    cudaFree(a->d_work);
    cudaFree(a->d_gH1);
    cudaFree(a->d_mpart);
    cudaFree(a->d_gH2);
    cudaFree(a->d_gp2);
    cudaFree(a->d_gm2);
    cudaFree(a->d_gin);
    cudaFree(a->d_partials);
    cudaFree(a->d_counter);
    cudaFree(a->d_slots);
    delete a;
}

mj_status adj_coef(mj_adjoint* a, const mj_dyn_params* p, DynCoef& c) {
    if (!p) return set_error(MJ_ERR_ARG, "null dynamics parameters");
    if (p->integrator != MJ_SIB) return set_error(MJ_ERR_UNSUPPORTED, "the adjoint differentiates the SIB integrator");
    std::memset(&c, 0, sizeof(c));  // the coefficients are part of the graph keys, padding included
    mj_status st = make_dyn_coef(p, a->plan, c);
    if (st != MJ_OK) return st;
    c.step_base = nullptr;
    return MJ_OK;
}

double* ckpt(const mj_adjoint* a, int k) { return a->d_ckpt + static_cast<int64_t>(k) * 3 * a->N; }

// One SIB stage of the forward map with explicit buffers: the plan's tiled
// kernels when a compile-time shape is active (the same arithmetic as
// mj_step), the generic stencil kernels otherwise.  The thermal draw is
// recomputed in the second stage.
void stage1(mj_plan* plan, const DynCoef& c, uint32_t step, const double* m, double* mb, cudaStream_t s) {
    if (plan->sp.shape != 0) {
        launch_tiled(plan, 4, c, m, nullptr, mb, nullptr, nullptr, DipView{nullptr, 0, 0, 0}, nullptr, step, s);
        return;
    }
    k_adj_f1<<<adj_grid(plan->sp), dim3(kABX, kABY), 0, s>>>(plan->sp, c, step, plan->d_bmap, m, mb);
}
void stage2(mj_plan* plan, const DynCoef& c, uint32_t step, const double* m, const double* mb, double* out,
            cudaStream_t s) {
    if (plan->sp.shape != 0) {
        launch_tiled(plan, 5, c, mb, m, out, nullptr, nullptr, DipView{nullptr, 0, 0, 0}, nullptr, step, s);
        return;
    }
    k_adj_f2<<<adj_grid(plan->sp), dim3(kABX, kABY), 0, s>>>(plan->sp, c, step, plan->d_bmap, m, mb, out);
}

// forward sweep from checkpoint 0 (already holding m_0) to checkpoint nseg
void forward_launches(mj_adjoint* a, const DynCoef& c, uint32_t step0, cudaStream_t s) {
    mj_plan* plan = a->plan;
    const int64_t n3 = 3 * a->N;
    double* mid = a->d_work + 2 * n3;
    const int E = a->every;
    for (int32_t k = 0; k < a->nsteps; ++k) {
        const double* src = (k % E == 0) ? ckpt(a, k / E) : a->d_work + (k % 2) * n3;
        const bool bound = ((k + 1) % E == 0) || (k + 1 == a->nsteps);
        double* dst = bound ? ckpt(a, (k + E) / E) : a->d_work + ((k + 1) % 2) * n3;
        const uint32_t step = step0 + static_cast<uint32_t>(k);
        stage1(plan, c, step, src, mid, s);
        stage2(plan, c, step, src, mid, dst, s);
    }
}

// backward sweep from d_gin (dL/dm_T) to d_g0, d_gterms and, if want_b, d_gb
void backward_launches(mj_adjoint* a, const DynCoef& c, uint32_t step0, bool want_b, cudaStream_t s) {
    mj_plan* plan = a->plan;
    const int64_t n3 = 3 * a->N;
    const int nt = plan_nterm(plan);
    const TermMasks M = term_masks(plan, nt);
    const dim3 grid = adj_grid(plan->sp), blk(kABX, kABY);
    double* gb = want_b ? a->d_gb : nullptr;
    if (gb) cudaMemsetAsync(gb, 0, sizeof(double) * n3, s);
    const int E = a->every;
    int slot = 0;
    bool first = true;
    for (int seg = a->nseg - 1; seg >= 0; --seg) {
        const int s0 = seg * E;
        const int len = std::min(E, a->nsteps - s0);
        // recompute the segment: m_n (slot 0 = the checkpoint) and mb of every step
        auto segm = [&](int k) -> double* { return k == 0 ? ckpt(a, seg) : a->d_segm + k * n3; };
        for (int k = 0; k < len; ++k) {
            const uint32_t step = step0 + static_cast<uint32_t>(s0 + k);
            stage1(plan, c, step, segm(k), a->d_segb + k * n3, s);
            if (k + 1 < len) stage2(plan, c, step, segm(k), a->d_segb + k * n3, segm(k + 1), s);
        }
        for (int k = len - 1; k >= 0; --k) {
            const uint32_t step = step0 + static_cast<uint32_t>(s0 + k);
            AdjReduce Ra{a->d_partials, a->d_counter, a->d_slots + static_cast<int64_t>(slot++) * kMaxTerms, a->nblocks};
            const CaArgs ca{step, first ? nullptr : a->d_gH1, first ? a->d_gin : a->d_mpart, segm(k),
                            a->d_segb + k * n3, nullptr, a->d_gH2, a->d_gp2, a->d_gm2, Ra};
            if (!tadj_dispatch(plan, c, M, &ca, nullptr, s))
                k_adj_ca<<<grid, blk, 0, s>>>(plan->sp, c, step, plan->d_bmap, plan->d_unit, M, ca.gH1, ca.mpart, ca.m,
                                              ca.mb, nullptr, a->d_gH2, a->d_gp2, a->d_gm2, Ra);
            first = false;
            AdjReduce Rb{a->d_partials, a->d_counter, a->d_slots + static_cast<int64_t>(slot++) * kMaxTerms, a->nblocks};
            const BArgs bb{step, a->d_gH2, a->d_gp2, a->d_gm2, segm(k), a->d_gH1, a->d_mpart, gb, Rb};
            if (!tadj_dispatch(plan, c, M, nullptr, &bb, s))
                k_adj_b<<<grid, blk, 0, s>>>(plan->sp, c, step, plan->d_bmap, plan->d_unit, M, a->d_gH2, a->d_gp2,
                                             a->d_gm2, segm(k), a->d_gH1, a->d_mpart, gb, Rb);
        }
    }
    // dL/dm_0 = mpart + W gH1 of step 0
    AdjReduce R0{nullptr, nullptr, nullptr, 0};
    const TermMasks M0 = term_masks(plan, 0);
    const CaArgs c0{0u, a->d_gH1, a->d_mpart, nullptr, nullptr, a->d_g0, nullptr, nullptr, nullptr, R0};
    if (!tadj_dispatch(plan, c, M0, &c0, nullptr, s))
        k_adj_ca<<<grid, blk, 0, s>>>(plan->sp, c, 0u, plan->d_bmap, plan->d_unit, M0, a->d_gH1, a->d_mpart, nullptr,
                                      nullptr, a->d_g0, nullptr, nullptr, nullptr, R0);
    if (nt > 0) k_adj_sum<<<1, kMaxTerms, 0, s>>>(a->d_slots, slot, nt, a->d_gterms);
}

// everything a sweep's launches depend on besides the buffers it owns
std::string sweep_key(const mj_adjoint* a, const DynCoef& c, uint32_t step0, int flags) {
    std::string k(reinterpret_cast<const char*>(&c), sizeof(c));
    k.append(reinterpret_cast<const char*>(&a->plan->sp), sizeof(StencilParams));
    const void* ptrs[2] = {a->plan->d_bmap, a->plan->d_unit};
    k.append(reinterpret_cast<const char*>(ptrs), sizeof(ptrs));
    k += "/" + std::to_string(step0) + "/" + std::to_string(flags);
    return k;
}

// replay `launches` as a CUDA graph on s, capturing it again when the key changed
template <class Fn>
mj_status run_sweep(mj_adjoint* a, cudaGraphExec_t& exec, std::string& cached, const std::string& key, Fn launches,
                    cudaStream_t s) {
    mj_status st;
    if (!a->cap && (st = cuda_status(cudaStreamCreateWithFlags(&a->cap, cudaStreamNonBlocking), "capture stream")) != MJ_OK)
        return st;
    if (!exec || cached != key) {
        if (exec) {
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
        if ((st = cuda_status(cudaStreamBeginCapture(a->cap, cudaStreamCaptureModeThreadLocal), "begin capture")) != MJ_OK)
            return st;
        launches(a->cap);
        cudaGraph_t g = nullptr;
        const cudaError_t launch_err = cudaGetLastError();
        const cudaError_t e = cudaStreamEndCapture(a->cap, &g);
        if (launch_err != cudaSuccess || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_status(launch_err != cudaSuccess ? launch_err : e, "adjoint capture");
        }
        const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            exec = nullptr;
            return cuda_status(ie, "adjoint graph instantiate");
        }
        cached = key;
    }
    return cuda_status(cudaGraphLaunch(exec, s), "adjoint graph launch");
}

}  // namespace
}  // namespace mj

using namespace mj;

extern "C" {

mj_status mj_plan_nterms(const mj_plan* plan, int32_t* n) {
    if (!plan || !n) return set_error(MJ_ERR_ARG, "null argument");
    *n = plan_nterm(plan);
    return MJ_OK;
}

mj_status mj_plan_set_terms(mj_plan* plan, const double* values) {
    if (!plan || !values) return set_error(MJ_ERR_ARG, "null argument");
    if (!plan->is_stencil) return set_error(MJ_ERR_UNSUPPORTED, "term values can be reset on stencil plans only");
    cudaSetDevice(plan->device);
    mj_status st = ensure_units(plan);
    if (st != MJ_OK) return st;
    const int nt = plan_nterm(plan);
    StencilParams sp = plan->sp;
    const int n_off = sp.n_off;
    for (int k = 0; k <= n_off; ++k) {
        double W[9];
        for (int q = 0; q < 9; ++q) {
            double s = 0.0;
            for (int t = 0; t < nt; ++t) s += values[t] * plan->unitW[(static_cast<size_t>(t) * (n_off + 1) + k) * 9 + q];
            W[q] = s;
        }
        if (k < n_off) {
            bool iso = W[0] == W[4] && W[0] == W[8];
            for (int q = 0; q < 9; ++q) {
                sp.W[k][q] = W[q];
                if (q != 0 && q != 4 && q != 8 && W[q] != 0.0) iso = false;
            }
            sp.iso[k] = iso ? 1 : 0;
        } else {
            sp.has_onsite = 0;
            for (int q = 0; q < 9; ++q) {
                sp.W0[q] = W[q];
                if (W[q] != 0.0) sp.has_onsite = 1;
            }
        }
    }
    // the offsets keep their order; re-derive the compile-time shape (isotropy may change)
    const int forced_generic = plan->sp.shape == 0 && plan->tiled_shape != 0;
    match_shape(sp);
    plan->tiled_shape = sp.shape;
    if (forced_generic) sp.shape = 0;
    plan->sp = sp;
    for (int t = 0; t < nt; ++t) {
        const int nJ = static_cast<int>(plan->termJ.size()), nD = static_cast<int>(plan->termD.size());
        if (t < nJ) plan->termJ[t].value = values[t];
        else if (t < nJ + nD) plan->termD[t - nJ].value = values[t];
        else plan->termK[t - nJ - nD].value = values[t];
    }
    drop_graph(plan);
    return MJ_OK;
}

mj_status mj_field_vjp(mj_plan* plan, const double* m, const double* v, double* g_m, double* g_terms, double* g_b,
                       void* stream) {
    if (!plan || !m || !v) return set_error(MJ_ERR_ARG, "null argument");
    if (!plan->is_stencil || plan->dip_on)
        return set_error(MJ_ERR_UNSUPPORTED, "the field VJP covers single-atom stencil plans without the dipolar term");
    cudaSetDevice(plan->device);
    mj_status st = ensure_units(plan);
    if (st != MJ_OK) return st;
    const int nt = g_terms ? plan_nterm(plan) : 0;
    if (nt > kMaxTerms) return set_error(MJ_ERR_UNSUPPORTED, "more than 8 coupling terms");
    const dim3 grid = adj_grid(plan->sp);
    const int nb = static_cast<int>(grid.x * grid.y * grid.z);
    if (nt > 0 && !plan->d_vjp_part) {  // allocated on first use
        if ((st = cuda_status(cudaMalloc(&plan->d_vjp_part, sizeof(double) * kMaxTerms * nb), "vjp scratch")) != MJ_OK)
            return st;
        if ((st = cuda_status(cudaMalloc(&plan->d_vjp_counter, sizeof(unsigned int) * 4), "vjp scratch")) != MJ_OK)
            return st;
        if ((st = cuda_status(cudaMemset(plan->d_vjp_counter, 0, sizeof(unsigned int) * 4), "vjp scratch")) != MJ_OK)
            return st;
    }
    AdjReduce R{plan->d_vjp_part, plan->d_vjp_counter, nt > 0 ? g_terms : nullptr, nb};
    k_field_vjp<<<grid, dim3(kABX, kABY), 0, static_cast<cudaStream_t>(stream)>>>(plan->sp, plan->d_unit,
                                                                                  term_masks(plan, nt), m, v, g_m,
                                                                                  g_b, R);
    return cuda_status(cudaGetLastError(), "k_field_vjp");
}

mj_status mj_adjoint_create(mj_plan* plan, int32_t nsteps, int32_t checkpoint_every, mj_adjoint** out) {
    if (!plan || !out || nsteps < 1 || checkpoint_every < 1) return set_error(MJ_ERR_ARG, "bad adjoint arguments");
    *out = nullptr;
    if (!plan->is_stencil || plan->dip_on)
        return set_error(MJ_ERR_UNSUPPORTED, "the adjoint covers single-atom stencil plans without the dipolar term");
    if (plan_nterm(plan) > kMaxTerms) return set_error(MJ_ERR_UNSUPPORTED, "more than 8 coupling terms");
    cudaSetDevice(plan->device);
    mj_status st = ensure_units(plan);
    if (st != MJ_OK) return st;
    mj_adjoint* a = new mj_adjoint();
    a->plan = plan;
    a->nsteps = nsteps;
    a->every = std::min(checkpoint_every, nsteps);
    a->nseg = (nsteps + a->every - 1) / a->every;
    a->N = plan->N;
    const dim3 grid = adj_grid(plan->sp);
    a->nblocks = static_cast<int>(grid.x * grid.y * grid.z);
    const size_t f3 = sizeof(double) * 3 * static_cast<size_t>(a->N);
    auto al = [&](auto** ptr, size_t bytes, const char* what) {
        return cuda_status(cudaMalloc(reinterpret_cast<void**>(ptr), bytes), what);
    };
    if ((st = al(&a->d_ckpt, f3 * (a->nseg + 1), "adjoint checkpoints")) != MJ_OK ||
        (st = al(&a->d_segm, f3 * a->every, "adjoint segment")) != MJ_OK ||
        (st = al(&a->d_segb, f3 * a->every, "adjoint segment")) != MJ_OK ||
        (st = al(&a->d_work, f3 * 3, "adjoint work")) != MJ_OK || (st = al(&a->d_gH1, f3, "adjoint")) != MJ_OK ||
        (st = al(&a->d_mpart, f3, "adjoint")) != MJ_OK || (st = al(&a->d_gH2, f3, "adjoint")) != MJ_OK ||
        (st = al(&a->d_gp2, f3, "adjoint")) != MJ_OK || (st = al(&a->d_gm2, f3, "adjoint")) != MJ_OK ||
        (st = al(&a->d_gin, f3, "adjoint")) != MJ_OK ||
        (st = al(&a->d_partials, sizeof(double) * kMaxTerms * a->nblocks, "adjoint partials")) != MJ_OK ||
        (st = al(&a->d_counter, sizeof(unsigned int) * 4, "adjoint counter")) != MJ_OK ||
        (st = al(&a->d_slots, sizeof(double) * kMaxTerms * 2 * static_cast<size_t>(nsteps), "adjoint slots")) != MJ_OK ||
        (st = al(&a->d_g0, f3, "adjoint")) != MJ_OK ||
        (st = al(&a->d_gterms, sizeof(double) * kMaxTerms, "adjoint")) != MJ_OK) {
        adjoint_free(a);
        return st;
    }
    cudaMemset(a->d_counter, 0, sizeof(unsigned int) * 4);
    if ((st = cuda_status(cudaDeviceSynchronize(), "adjoint create")) != MJ_OK) {
        adjoint_free(a);
        return st;
    }
    *out = a;
    return MJ_OK;
}

mj_status mj_adjoint_destroy(mj_adjoint* a) {
    if (a) {
        cudaSetDevice(a->plan->device);
        adjoint_free(a);
    }
    return MJ_OK;
}

mj_status mj_adjoint_forward(mj_adjoint* a, const mj_dyn_params* p, const double* m0, double* mT, void* stream) {
    if (!a || !p || !m0) return set_error(MJ_ERR_ARG, "null argument");
    mj_plan* plan = a->plan;
    cudaSetDevice(plan->device);
    DynCoef c;
    mj_status st = adj_coef(a, p, c);
    if (st != MJ_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t f3 = sizeof(double) * 3 * static_cast<size_t>(a->N);
    if ((st = cuda_status(cudaMemcpyAsync(ckpt(a, 0), m0, f3, cudaMemcpyDeviceToDevice, s), "adjoint m0")) != MJ_OK)
        return st;
    const uint32_t step0 = p->step0;
    st = run_sweep(a, a->gfwd, a->kfwd, sweep_key(a, c, step0, 0),
                   [&](cudaStream_t cs) { forward_launches(a, c, step0, cs); }, s);
    if (st != MJ_OK) return st;
    if (mT && (st = cuda_status(cudaMemcpyAsync(mT, ckpt(a, a->nseg), f3, cudaMemcpyDeviceToDevice, s), "adjoint mT")) !=
                  MJ_OK)
        return st;
    a->prm = *p;
    a->have_forward = true;
    return MJ_OK;
}

mj_status mj_adjoint_backward(mj_adjoint* a, const double* gT, double* g0, double* g_terms, double* g_b, void* stream) {
    if (!a || !gT || !g0) return set_error(MJ_ERR_ARG, "null argument");
    if (!a->have_forward) return set_error(MJ_ERR_ARG, "mj_adjoint_backward needs a forward run first");
    mj_plan* plan = a->plan;
    cudaSetDevice(plan->device);
    DynCoef c;
    mj_status st = adj_coef(a, &a->prm, c);
    if (st != MJ_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t f3 = sizeof(double) * 3 * static_cast<size_t>(a->N);
    const int nt = plan_nterm(plan);
    const bool want_b = g_b != nullptr;
    if (want_b && !a->d_gb && (st = cuda_status(cudaMalloc(&a->d_gb, f3), "adjoint g_b")) != MJ_OK) return st;
    // dL/dm_T enters as the "partial" of a step with no W gH1 term
    if ((st = cuda_status(cudaMemcpyAsync(a->d_gin, gT, f3, cudaMemcpyDeviceToDevice, s), "adjoint gT")) != MJ_OK)
        return st;
    const uint32_t step0 = a->prm.step0;
    st = run_sweep(a, a->gbwd, a->kbwd, sweep_key(a, c, step0, want_b ? 1 : 0),
                   [&](cudaStream_t cs) { backward_launches(a, c, step0, want_b, cs); }, s);
    if (st != MJ_OK) return st;
    if ((st = cuda_status(cudaMemcpyAsync(g0, a->d_g0, f3, cudaMemcpyDeviceToDevice, s), "adjoint g0")) != MJ_OK)
        return st;
    if (g_terms && nt > 0 &&
        (st = cuda_status(cudaMemcpyAsync(g_terms, a->d_gterms, sizeof(double) * nt, cudaMemcpyDeviceToDevice, s),
                          "adjoint g_terms")) != MJ_OK)
        return st;
    if (want_b && (st = cuda_status(cudaMemcpyAsync(g_b, a->d_gb, f3, cudaMemcpyDeviceToDevice, s), "adjoint g_b")) != MJ_OK)
        return st;
    return MJ_OK;
}

}  // extern "C"
