// Device helpers shared by the field, step, batch and adjoint kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mj_internal.hpp"

namespace mj {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11) and Box-Muller normals.  Counter = (site, step, stream,
// 0), key = the 64-bit seed: one block per site and step, whose four 32-bit
// words give the three normals (r1 cos t1, r1 sin t1, r2 cos t2) with
// r = sqrt(-2 ln u), u = (w0 + 1/2) 2^-32 and (w2 + 1/2) 2^-32, and
// t = 2 pi (w + 1/2) 2^-32 for w1 and w3.
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

// Philox4x32-10 with the ten round keys precomputed (keys[2r], keys[2r+1]);
// each round's two products as one 32 x 32 -> 64-bit multiply (low and high
// words of the same product).
__device__ __forceinline__ void philox10k(uint32_t c[4], const uint32_t* keys) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(M0) * c[0], p1 = static_cast<uint64_t>(M1) * c[2];
        const uint32_t lo0 = static_cast<uint32_t>(p0), hi0 = static_cast<uint32_t>(p0 >> 32);
        const uint32_t lo1 = static_cast<uint32_t>(p1), hi1 = static_cast<uint32_t>(p1 >> 32);
        const uint32_t n0 = hi1 ^ c[1] ^ keys[2 * r];
        const uint32_t n2 = hi0 ^ c[3] ^ keys[2 * r + 1];
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

// Two independent blocks through the same rounds (the round keys read once,
// the two dependency chains interleaved): the same words as two philox10k calls.
__device__ __forceinline__ void philox10k_x2(uint32_t a[4], uint32_t b[4], const uint32_t* keys) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t k0 = keys[2 * r], k1 = keys[2 * r + 1];
        const uint64_t pa0 = static_cast<uint64_t>(M0) * a[0], pa1 = static_cast<uint64_t>(M1) * a[2];
        const uint64_t pb0 = static_cast<uint64_t>(M0) * b[0], pb1 = static_cast<uint64_t>(M1) * b[2];
        const uint32_t na0 = static_cast<uint32_t>(pa1 >> 32) ^ a[1] ^ k0;
        const uint32_t na2 = static_cast<uint32_t>(pa0 >> 32) ^ a[3] ^ k1;
        const uint32_t nb0 = static_cast<uint32_t>(pb1 >> 32) ^ b[1] ^ k0;
        const uint32_t nb2 = static_cast<uint32_t>(pb0 >> 32) ^ b[3] ^ k1;
        a[0] = na0;
        a[1] = static_cast<uint32_t>(pa1);
        a[2] = na2;
        a[3] = static_cast<uint32_t>(pa0);
        b[0] = nb0;
        b[1] = static_cast<uint32_t>(pb1);
        b[2] = nb2;
        b[3] = static_cast<uint32_t>(pb0);
    }
}

// Table-driven FP64 log and sin/cos (our own evaluation, the same arithmetic
// as the oracle's; every step is one rounded operation or an explicit fma):
// tab[2i], tab[2i+1]         (sin, cos)(2 pi (i + 1/2)/1024),  i = 0..1023
// tab[2048+2j], tab[2049+2j] (1/F_j, ln F_j), F_j = 1 + (j + 1/2)/1024, j = 0..1023
//   ln u = e ln2 + ln F + ln(1 + r), u = 2^e m, m in [1, 2), j = the top ten
//   mantissa bits, r = m/F - 1 (|r| < 1/2049), ln(1 + r) to r^4 (error below
//   6e-18); ln u within 3 ulp plus 3e-16 absolute (above u = 1/2 it cancels
//   against -ln 2);
//   sin/cos(a_i + x), |x| <= pi/1024, sin x to x^5 and cos x - 1 to x^4 (errors
//   below 1.2e-18); absolute error below 3e-16.
constexpr double kLn2 = 0.6931471805599453;                 // ln 2
constexpr double kTwoPiOver2p32 = 1.4629180792671596e-09;   // 2 pi / 2^32
constexpr double kPiOver2p32 = 7.314590396335798e-10;       // pi / 2^32

// 53-bit uniform in [0, 1) from two words (the parallel-tempering acceptance draw)
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    const uint64_t k = (static_cast<uint64_t>(a >> 5) << 26) | static_cast<uint64_t>(b >> 6);
    return static_cast<double>(k) * (1.0 / 9007199254740992.0);
}

// u = (w + 1/2) 2^-32 in (0, 1), exact in double
__device__ __forceinline__ double u32_half(uint32_t w) { return fma(static_cast<double>(w), 0x1p-32, 0x1p-33); }

__device__ __forceinline__ double tab_log(double u, const double* __restrict__ tab) {
    const int hi = __double2hiint(u);
    const int e = ((hi >> 20) & 0x7ff) - 1023;
    const int j = (hi >> 10) & 0x3ff;
    const double m = __hiloint2double((hi & 0x000fffff) | 0x3ff00000, __double2loint(u));
    const double2 t = __ldg(reinterpret_cast<const double2*>(tab + 2048) + j);
    const double r = fma(m, t.x, -1.0);
    const double p = fma(fma(r, -0.25, 1.0 / 3.0), r, -0.5);
    const double l1p = fma(r * r, p, r);
    return fma(static_cast<double>(e), kLn2, t.y + l1p);
}

// sin and cos of 2 pi (w + 1/2) 2^-32: table point a_i = 2 pi (i + 1/2)/1024 with
// i = w >> 22, remainder x = 2 pi ((w mod 2^22) - 2^21 + 1/2) 2^-32
__device__ __forceinline__ void sincos2pi_word(uint32_t w, const double* __restrict__ tab, double* s, double* c) {
    const int i = static_cast<int>(w >> 22);
    const int d = static_cast<int>(w & 0x3fffffu) - 2097152;
    const double x = fma(static_cast<double>(d), kTwoPiOver2p32, kPiOver2p32);
    const double x2 = x * x;
    const double sx = fma(x * x2, fma(x2, 1.0 / 120.0, -1.0 / 6.0), x);
    const double cm = x2 * fma(x2, 1.0 / 24.0, -0.5);
    const double2 t = __ldg(reinterpret_cast<const double2*>(tab) + i);
    *s = t.x + fma(t.x, cm, t.y * sx);
    *c = t.y + fma(t.y, cm, -(t.x * sx));
}

// The three normals of one Philox block's words: (r1 cos t1, r1 sin t1, r2 cos t2)
__device__ __forceinline__ double3 normals_of_block(const uint32_t c[4], const double* __restrict__ tab) {
    const double r1 = sqrt(-2.0 * tab_log(u32_half(c[0]), tab));
    const double r2 = sqrt(-2.0 * tab_log(u32_half(c[2]), tab));
    double s1, c1, s2, c2;
    sincos2pi_word(c[1], tab, &s1, &c1);
    sincos2pi_word(c[3], tab, &s2, &c2);
    return make_double3(r1 * c1, r1 * s1, r2 * c2);
}

// N(0,1) triple of one site and step from one Philox block, counter = (site,
// step, stream, 0)
__device__ __forceinline__ double3 philox_normals_tab(const uint32_t* keys, const double* __restrict__ tab,
                                                      uint32_t step, uint32_t stream, uint32_t site) {
    uint32_t c[4] = {site, step, stream, 0u};
    philox10k(c, keys);
    return normals_of_block(c, tab);
}

// The normals of two sites of one step and stream together (the words and
// normals of two philox_normals_tab calls).
__device__ __forceinline__ void philox_normals_x2(const uint32_t* keys, const double* __restrict__ tab, uint32_t step,
                                                  uint32_t stream, uint32_t site0, uint32_t site1, double3& z0,
                                                  double3& z1) {
    uint32_t a[4] = {site0, step, stream, 0u};
    uint32_t b[4] = {site1, step, stream, 0u};
    philox10k_x2(a, b, keys);
    z0 = normals_of_block(a, tab);
    z1 = normals_of_block(b, tab);
}

// The same from the 64-bit seed (round keys derived here)
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

// The Philox thermal fields of two sites of one step together (the words and
// normals of two thermal_field calls).
__device__ __forceinline__ void thermal_field_x2(const DynCoef& C, uint32_t step, int64_t i0, int64_t i1, double3& b0,
                                                 double3& b1) {
    if (C.step_base) step += *C.step_base;
    double3 za, zb;
    philox_normals_x2(C.keys, C.noise_tab, step, C.stream_id, static_cast<uint32_t>(i0), static_cast<uint32_t>(i1), za,
                      zb);
    b0 = make_double3(C.sigma * za.x, C.sigma * za.y, C.sigma * za.z);
    b1 = make_double3(C.sigma * zb.x, C.sigma * zb.y, C.sigma * zb.z);
}

// ---------------------------------------------------------------------------
// A step's new spin: a non-finite component sets kStatusNonFinite in the plan's
// status word (mj_plan_check_status then reports MJ_ERR_NAN).
__device__ __forceinline__ void flag_nonfinite(int* status, double3 v) {
    if (!isfinite(v.x + v.y + v.z) && status) atomicOr(status, kStatusNonFinite);
}

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

__device__ __forceinline__ void st_pad(const DipPad& d, int x, int y, int z, double3 v) {
    const int64_t q = x + static_cast<int64_t>(d.px) * y + d.zs * z;
    d.p[q] = v.x;
    d.p[d.cs + q] = v.y;
    d.p[2 * d.cs + q] = v.z;
}
__device__ __forceinline__ double3 ld_dip(const DipView& v, int x, int y, int z) {
    const int64_t q = x + static_cast<int64_t>(v.px) * y + v.zs * z;
    return make_double3(__ldg(v.h + q), __ldg(v.h + v.cs + q), __ldg(v.h + 2 * v.cs + q));
}

// 1/|v| and |v| from n2 = |v|^2 for the vectors of the step, unit spins or the
// midpoint of two (n2 = 1 - O(|h|^2)): with d = n2 - 1, |d| < 2^-20, the series
// 1 + d (-1/2 + 3/8 d) and 1 + d (1/2 - d/8) (truncation below 3e-19 and 4e-20,
// below a rounding), else rsqrt / sqrt.  inv_norm returns 1 for n2 <= 1e-16
// (the 1e-8 guard of vector.f90:76-85).
__device__ __forceinline__ double inv_norm(double n2) {
    const double d = n2 - 1.0;
    if (fabs(d) < 0x1p-20) return fma(d, fma(d, 0.375, -0.5), 1.0);
    return n2 > 1e-16 ? rsqrt(n2) : 1.0;
}
__device__ __forceinline__ double norm_of(double n2) {
    const double d = n2 - 1.0;
    if (fabs(d) < 0x1p-20) return fma(d, fma(d, -0.125, 0.5), 1.0);
    return sqrt(n2);
}

// 2/(1 + q), q = |h|^2 of a SIB stage: 2 (1 - q + q^2 - q^3) for q < 2^-14
// (truncation below 1.4e-17 relative), else the division
__device__ __forceinline__ double cayley_scale(double q) {
    if (q < 0x1p-14) return fma(q, fma(q, fma(q, -2.0, 2.0), -2.0), 2.0);
    return 2.0 / (1.0 + q);
}

// Matjes LLG right-hand side (solvers/propagator.f90:13-58):
// D = -[m^ x B + alpha m^ x (m^ x B)] / (1 + alpha^2), m^ = m/|m| when |m| > 1e-8.
__device__ __forceinline__ double3 llg_rhs(double3 B, double3 m, double alpha, double inv_den) {
    const double inv = inv_norm(dot(m, m));
    const double3 mn = make_double3(m.x * inv, m.y * inv, m.z * inv);
    const double3 t = cross(mn, B);
    const double3 l = make_double3(B.x + alpha * t.x, B.y + alpha * t.y, B.z + alpha * t.z);
    const double3 o = cross(mn, l);
    return make_double3(-o.x * inv_den, -o.y * inv_den, -o.z * inv_den);
}

// Projection onto the old norm (solvers/solver.f90:113-116), |t| > 1e-8 guard.
__device__ __forceinline__ double3 project(double3 t, double3 m) {
    const double nt2 = dot(t, t);
    if (!(nt2 > 1e-16)) return m;
    const double s = norm_of(dot(m, m)) * inv_norm(nt2);
    return make_double3(t.x * s, t.y * s, t.z * s);
}

// SIB stage (Mentink et al., J. Phys.: Condens. Matter 22, 176001 (2010)):
// y = m + ((m + y)/2) x a,  h = a/2 = hc (H + alpha p^ x H), hc = -dt/(2 hbar (1+alpha^2)).
// Closed form (the Cayley transform of the rotation): y = m + 2/(1+|h|^2) (u + u x h),
// u = m x h  (|y| = |m|).
// MID: the predictor's midpoint (m + y)/2 = m + c/2 (u + u x h) instead of y.
template <bool MID = false>
__device__ __forceinline__ double3 sib_solve(double3 m, double3 p, double3 H, double alpha, double hc) {
    // h = hc H + (hc alpha / |p|) p x H: the normalisation folded into one scalar
    const double sa = hc * alpha * inv_norm(dot(p, p));
    const double3 pxh = cross(p, H);
    const double3 h = make_double3(fma(sa, pxh.x, hc * H.x), fma(sa, pxh.y, hc * H.y), fma(sa, pxh.z, hc * H.z));
    const double3 u = cross(m, h);
    const double3 w = cross(u, h);
    double c = cayley_scale(dot(h, h));
    if constexpr (MID) c = 0.5 * c;
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

// ---------------------------------------------------------------------------
// The six GNEB path sums of one site (GNEB/tangent.f90, gneb_utils.f90):
// A = P(m_{r+1} - m), B = P(m - m_{r-1}) (zero at the ends), |A|^2, A.B, |B|^2,
// F.A, F.B, squared angle to image r + 1.  The same arithmetic as the batch's
// GNEB field pass.
__device__ __forceinline__ void gneb_path_terms(double3 m0, double3 mp, double3 mm, bool up, double3 F, double (&g)[6]) {
    double3 u = make_double3(mp.x - m0.x, mp.y - m0.y, mp.z - m0.z);
    double3 w = make_double3(m0.x - mm.x, m0.y - mm.y, m0.z - mm.z);
    const double du = dot(u, m0), dw = dot(w, m0);
    u = make_double3(u.x - du * m0.x, u.y - du * m0.y, u.z - du * m0.z);
    w = make_double3(w.x - dw * m0.x, w.y - dw * m0.y, w.z - dw * m0.z);
    g[0] += dot(u, u);
    g[1] += dot(u, w);
    g[2] += dot(w, w);
    g[3] += dot(F, u);
    g[4] += dot(F, w);
    if (up) {
        const double3 c = cross(m0, mp);
        const double l = atan2(sqrt(dot(c, c)), dot(m0, mp));
        g[5] += l * l;
    }
}

}  // namespace mj
