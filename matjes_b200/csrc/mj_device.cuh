// Device helpers shared by the field, step, batch and adjoint kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mj_internal.hpp"

namespace mj {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11) and Box-Muller normals.  Counter = (site, step, stream,
// call), key = the 64-bit seed.  Two calls give two Box-Muller pairs of 53-bit
// uniforms: (r1 cos t1, r1 sin t1, r2 cos t2).
__device__ __forceinline__ void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        const uint32_t lo0 = M0 * c[0], hi0 = __umulhi(M0, c[0]);
        const uint32_t lo1 = M1 * c[2], hi1 = __umulhi(M1, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

__device__ __forceinline__ double u53_open(uint32_t a, uint32_t b) {
    const uint64_t k = (static_cast<uint64_t>(a >> 5) << 26) | static_cast<uint64_t>(b >> 6);
    return static_cast<double>(k + 1) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    const uint64_t k = (static_cast<uint64_t>(a >> 5) << 26) | static_cast<uint64_t>(b >> 6);
    return static_cast<double>(k) * (1.0 / 9007199254740992.0);
}

// Philox4x32-10 with the ten round keys precomputed (keys[2r], keys[2r+1]).
__device__ __forceinline__ void philox10k(uint32_t c[4], const uint32_t* keys) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = M0 * c[0], hi0 = __umulhi(M0, c[0]);
        const uint32_t lo1 = M1 * c[2], hi1 = __umulhi(M1, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ keys[2 * r];
        const uint32_t n2 = hi0 ^ c[3] ^ keys[2 * r + 1];
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

// Table-driven FP64 log and sin/cos of 2 pi u (our own evaluation, the same
// arithmetic as the oracle's): tab[0..511] = (sin, cos)(2 pi i/256) pairs,
// tab[512..767] = (1/F, ln F) pairs for F = (j + 96)/128 (j = 0..96 used).
//   ln u = e ln2 + ln F + ln(1 + r), mantissa m in [0.75, 1.5), F the nearest
//   multiple of 1/128, r = (m - F)/F, |r| <= 1/192, series to r^7;
//   2 pi u = 2 pi i/256 + x, |x| < pi/128, Taylor sin to x^7 and cos to x^8.
constexpr double kLn2 = 0.6931471805599453;        // ln 2
constexpr double kPiOver128 = 0.02454369260617026;  // pi / 128

__device__ __forceinline__ double tab_log(double u, const double* __restrict__ tab) {
    const long long b = __double_as_longlong(u);
    int e = static_cast<int>((b >> 52) & 0x7ff) - 1023;
    double m = __longlong_as_double((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    if (m >= 1.5) {  // centre the mantissa in [0.75, 1.5): no cancellation against e ln2 near u = 1
        m *= 0.5;
        e += 1;
    }
    const int j = static_cast<int>(m * 128.0 + 0.5);  // nearest F = j/128, j = 96..192
    const double F = static_cast<double>(j) * (1.0 / 128.0);
    const double2 t = __ldg(reinterpret_cast<const double2*>(tab + 512) + (j - 96));
    const double r = (m - F) * t.x;
    double p = fma(r, 1.0 / 7.0, -1.0 / 6.0);
    p = fma(p, r, 1.0 / 5.0);
    p = fma(p, r, -0.25);
    p = fma(p, r, 1.0 / 3.0);
    p = fma(p, r, -0.5);
    const double l1p = fma(r * r, p, r);
    return fma(static_cast<double>(e), kLn2, t.y + l1p);
}

__device__ __forceinline__ void tab_sincos2pi(double u, const double* __restrict__ tab, double* s, double* c) {
    const double t = u * 256.0;
    const int i = static_cast<int>(t);
    const double x = (t - static_cast<double>(i)) * kPiOver128;
    const double x2 = x * x;
    double ps = fma(x2, -1.0 / 5040.0, 1.0 / 120.0);
    ps = fma(ps, x2, -1.0 / 6.0);
    const double sx = fma(x * x2, ps, x);
    double pc = fma(x2, 1.0 / 40320.0, -1.0 / 720.0);
    pc = fma(pc, x2, 1.0 / 24.0);
    pc = fma(pc, x2, -0.5);
    const double cm = x2 * pc;
    const double2 sc = __ldg(reinterpret_cast<const double2*>(tab) + i);
    *s = sc.x + fma(sc.x, cm, sc.y * sx);
    *c = sc.y + fma(sc.y, cm, -(sc.x * sx));
}

// N(0,1) triple of one site and step: two Box-Muller pairs from two Philox
// blocks, counter = (site, step, stream, call), 53-bit uniforms.
__device__ __forceinline__ double3 philox_normals_tab(const uint32_t* keys, const double* __restrict__ tab,
                                                      uint32_t step, uint32_t stream, uint32_t site) {
    uint32_t c[4] = {site, step, stream, 0u};
    philox10k(c, keys);
    uint32_t d[4] = {site, step, stream, 1u};
    philox10k(d, keys);
    const double r1 = sqrt(-2.0 * tab_log(u53_open(c[0], c[1]), tab));
    const double r2 = sqrt(-2.0 * tab_log(u53_open(d[0], d[1]), tab));
    double s1, c1, s2, c2;
    tab_sincos2pi(u53(c[2], c[3]), tab, &s1, &c1);
    tab_sincos2pi(u53(d[2], d[3]), tab, &s2, &c2);
    return make_double3(r1 * c1, r1 * s1, r2 * c2);
}

__device__ __forceinline__ double3 philox_normals(uint64_t seed, uint32_t step, uint32_t stream, uint32_t site,
                                                  const double* __restrict__ tab) {
    uint32_t keys[20];
    uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        keys[2 * r] = k0;
        keys[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return philox_normals_tab(keys, tab, step, stream, site);
}

// Thermal field b = sigma * N(0,1) (dynamics/spindynamics.f90:268-272): Philox
// in-kernel, or read from an injected N(0,1) buffer laid out [nbuf][3][N].
__device__ __forceinline__ double3 thermal_field(const DynCoef& C, uint32_t step, int64_t i, int64_t N) {
    if (C.step_base) step += *C.step_base;
    if (C.noise == MJ_NOISE_PHILOX) {
        const double3 z = philox_normals_tab(C.keys, C.noise_tab, step, C.stream_id, static_cast<uint32_t>(i));
        return make_double3(C.sigma * z.x, C.sigma * z.y, C.sigma * z.z);
    }
    const double* buf = C.inject + static_cast<int64_t>(step % static_cast<uint32_t>(C.inject_nbuf)) * 3 * N;
    return make_double3(C.sigma * __ldg(buf + i), C.sigma * __ldg(buf + N + i), C.sigma * __ldg(buf + 2 * N + i));
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ double3 cross(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ double3 ld3(const double* __restrict__ m, int64_t i, int64_t N) {
    return make_double3(__ldg(m + i), __ldg(m + N + i), __ldg(m + 2 * N + i));
}
__device__ __forceinline__ void st3(double* m, int64_t i, int64_t N, double3 v) {
    m[i] = v.x;
    m[N + i] = v.y;
    m[2 * N + i] = v.z;
}

__device__ __forceinline__ double3 ld_dip(const DipView& v, int x, int y, int z) {
    const int64_t q = x + static_cast<int64_t>(v.px) * y + v.zs * z;
    return make_double3(__ldg(v.h + q), __ldg(v.h + v.cs + q), __ldg(v.h + 2 * v.cs + q));
}

// Matjes LLG right-hand side (solvers/propagator.f90:13-58):
// D = -[m^ x B + alpha m^ x (m^ x B)] / (1 + alpha^2), m^ = m/|m| when |m| > 1e-8.
__device__ __forceinline__ double3 llg_rhs(double3 B, double3 m, double alpha, double inv_den) {
    const double n2 = dot(m, m);
    double3 mn = m;
    if (n2 > 1e-16) {
        const double inv = rsqrt(n2);
        mn = make_double3(m.x * inv, m.y * inv, m.z * inv);
    }
    const double3 t = cross(mn, B);
    const double3 l = make_double3(B.x + alpha * t.x, B.y + alpha * t.y, B.z + alpha * t.z);
    const double3 o = cross(mn, l);
    return make_double3(-o.x * inv_den, -o.y * inv_den, -o.z * inv_den);
}

// Projection onto the old norm (solvers/solver.f90:113-116), |t| > 1e-8 guard.
__device__ __forceinline__ double3 project(double3 t, double3 m) {
    const double nt = sqrt(dot(t, t));
    if (!(nt > 1e-8)) return m;
    const double s = sqrt(dot(m, m)) / nt;
    return make_double3(t.x * s, t.y * s, t.z * s);
}

// SIB stage (Mentink et al., J. Phys.: Condens. Matter 22, 176001 (2010)):
// y = m + ((m + y)/2) x a,  h = a/2 = hc (H + alpha p^ x H), hc = -dt/(2 hbar (1+alpha^2)).
// Closed form (the Cayley transform of the rotation): y = m + 2/(1+|h|^2) (u + u x h),
// u = m x h  (|y| = |m|).
__device__ __forceinline__ double3 sib_solve(double3 m, double3 p, double3 H, double alpha, double hc) {
    const double np2 = dot(p, p);
    double3 pn = p;
    if (np2 > 1e-16) {
        const double inv = rsqrt(np2);
        pn = make_double3(p.x * inv, p.y * inv, p.z * inv);
    }
    const double3 pxh = cross(pn, H);
    const double3 h = make_double3(hc * (H.x + alpha * pxh.x), hc * (H.y + alpha * pxh.y), hc * (H.z + alpha * pxh.z));
    const double3 u = cross(m, h);
    const double3 w = cross(u, h);
    const double c = 2.0 / (1.0 + dot(h, h));
    return make_double3(fma(c, u.x + w.x, m.x), fma(c, u.y + w.y, m.y), fma(c, u.z + w.z, m.z));
}

// ---------------------------------------------------------------------------
struct FieldOut {
    double3 B;     // real-space field (MM + Zeeman)
    double3 Bzee;  // Zeeman part
};

// Per-site energy (energy_distrib, left-assigned; hamiltonian_collection.f90:332-363):
// E_i = m.(H m)_i + E_zee,i with (H m)_i = -B_mm/2 for the symmetric combined MM
// matrix, and the dipolar term doubled as in fft_ham_base.f90:247-256.
__device__ __forceinline__ double site_energy(const FieldOut& f, double3 m, double3 Hd) {
    const double3 Bmm = make_double3(f.B.x - f.Bzee.x, f.B.y - f.Bzee.y, f.B.z - f.Bzee.z);
    return -0.5 * dot(m, Bmm) - dot(m, f.Bzee) + 2.0 * dot(m, Hd);
}
// Contribution of one site to H%energy (dipolar counted once, fft_ham_base.f90:258-267).
__device__ __forceinline__ double total_energy_part(const FieldOut& f, double3 m, double3 Hd) {
    const double3 Bmm = make_double3(f.B.x - f.Bzee.x, f.B.y - f.Bzee.y, f.B.z - f.Bzee.z);
    return -0.5 * dot(m, Bmm) - dot(m, f.Bzee) + dot(m, Hd);
}

// ---------------------------------------------------------------------------
// Deterministic grid reduction of NV doubles, in two halves that a caller may
// also use apart: block_partials writes one partial per block (warp sums in
// lane order, warps in order), ordered_sum adds nblocks partials in a fixed
// order (thread-strided sums, warp shuffles, warps in order).  grid_reduce does
// both in one launch: the last block to take a ticket sums the partials and
// re-arms the ticket counter.  Blocks of at most 256 threads.
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double* partials, int nblocks, int bid) {
    __shared__ double wsum_p[NV][8];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double e = v[q];
        for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
        if (lane == 0) wsum_p[q][wid] = e;
    }
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0.0;
            for (int w = 0; w < nthr / 32; ++w) s += wsum_p[q][w];
            partials[static_cast<int64_t>(q) * nblocks + bid] = s;
        }
    }
}

template <int NV>
__device__ void ordered_sum(const double* partials, int nblocks, double* out) {
    __shared__ double wsum_o[NV][8];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nthr = blockDim.x * blockDim.y;
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0.0;
        for (int b = tid; b < nblocks; b += nthr) s += __ldcg(partials + static_cast<int64_t>(q) * nblocks + b);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        __syncthreads();
        if (lane == 0) wsum_o[q][wid] = s;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < nthr / 32; ++w) t += wsum_o[q][w];
            out[q] = t;
        }
    }
}

template <int NV>
__device__ void grid_reduce(double (&v)[NV], double* partials, unsigned int* counter, double* out, int nblocks) {
    __shared__ bool last;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_partials<NV>(v, partials, nblocks, bid);
    if (tid == 0) {
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == static_cast<unsigned int>(nblocks - 1));
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    ordered_sum<NV>(partials, nblocks, out);
    if (tid == 0) *counter = 0u;
}

}  // namespace mj
