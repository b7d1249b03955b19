// Metropolis single-spin moves (Metropolis-MC/MCstep.f90) shared by the
// single-lattice sweeps (mj_mc.cu) and the batched replicas (mj_batch.cu).
//
// A move of site i in sweep t draws Philox4x32-10 counter (i, t, stream,
// 0x4D43) under the key of the seed: words 0 and 1 drive the proposal, word 2
// the acceptance test, each turned into a uniform in (0, 1) as (w + 0.5) 2^-32.
// Proposals (track_value.f90 sample_*): the cone of sphereft (paratemp-MC/
// sampling.f90:9-62), the Ising flip, under- and over-relaxation from the
// site's field (relaxationtype.f90).  The energy change is that of
// energy_single:
//   dE = -(s' - s).P - (s'^T W0 s' - s^T W0 s)/2 - (s' - s).(zc b)
// with P the pair field of the neighbours and W0 the on-site tensor; the move
// is taken when dE < 0 or when the uniform is below exp(max(-dE/kT, -200))
// (MCstep.f90:75-89).
#pragma once

#include <type_traits>
#include <utility>
#include <vector>

#include "mj_shapes.hpp"
#include "mj_stencil.cuh"

namespace mj {
namespace {

constexpr uint32_t kMcTag = 0x4D43u;  // "MC"

__device__ __forceinline__ double u32_open(uint32_t w) { return (static_cast<double>(w) + 0.5) * (1.0 / 4294967296.0); }

// sphereft: a direction in the cone of half-angle `cone` about s; sin and cos of
// phi = 2 pi (w2 + 1/2) 2^-32 from the tables of the thermal draw
// (sincos2pi_word, absolute error below 3e-16)
__device__ __forceinline__ double3 cone_proposal(double3 s, double cos_cone, double u1, uint32_t w2,
                                                 const double* __restrict__ tab) {
    const double ct = u1 + cos_cone * (1.0 - u1);
    const double st = sqrt(1.0 - ct * ct);
    const double cti = s.z;
    const double rxy2 = s.x * s.x + s.y * s.y;
    const double sti = sqrt(rxy2);
    double cpi = 1.0, spi = 0.0;
    if (!(rxy2 < 0.00001)) {
        const double inv = 1.0 / sti;
        cpi = s.x * inv;
        spi = s.y * inv;
    }
    double sph, cph;
    sincos2pi_word(w2, tab, &sph, &cph);
    const double t = st * sph * cti + ct * sti;
    const double3 n = make_double3(-st * cph * spi + t * cpi, st * cph * cpi + t * spi, -st * sph * sti + ct * cti);
    const double inv_n = 1.0 / sqrt(dot(n, n));
    return make_double3(n.x * inv_n, n.y * inv_n, n.z * inv_n);
}

// periodic neighbour k of (x, y, z) on a lattice of sizes (Lx, Ly, Lz)
__device__ __forceinline__ bool neighbour_in(const StencilParams& P, int Lx, int Ly, int Lz, int x, int y, int z,
                                             int k, int64_t& j) {
    int nx = x + P.off[k][0], ny = y + P.off[k][1], nz = z + P.off[k][2];
    if (nx < 0 || nx >= Lx) {
        if (!P.periodic[0]) return false;
        nx = wrap(nx, Lx);
    }
    if (ny < 0 || ny >= Ly) {
        if (!P.periodic[1]) return false;
        ny = wrap(ny, Ly);
    }
    if (nz < 0 || nz >= Lz) {
        if (!P.periodic[2]) return false;
        nz = wrap(nz, Lz);
    }
    j = nx + static_cast<int64_t>(Lx) * (ny + static_cast<int64_t>(Ly) * nz);
    return true;
}

// one compile-time offset k of shape S added to the pair field b
template <class S, int k>
__device__ __forceinline__ void pair_term(const StencilParams& P, const double* __restrict__ m, int64_t Ntot, int Lx,
                                          int Ly, int x, int y, int64_t layer, double3& b) {
    constexpr int dx = S::DX[k], dy = S::DY[k];
    int nx = x + dx, ny = y + dy;
    if (nx < 0 || nx >= Lx) {
        if (!P.periodic[0]) return;
        nx = wrap(nx, Lx);
    }
    if (ny < 0 || ny >= Ly) {
        if (!P.periodic[1]) return;
        ny = wrap(ny, Ly);
    }
    const double3 v = ld3(m, layer + nx + static_cast<int64_t>(Lx) * ny, Ntot);
    if constexpr (S::ISO[k] != 0) {
        const double w = P.W[k][0];
        b = make_double3(fma(w, v.x, b.x), fma(w, v.y, b.y), fma(w, v.z, b.z));
    } else {
        b = mat3(P.W[k], v, b);
    }
}

template <class S, int... Kk>
__device__ __forceinline__ void pair_terms(const StencilParams& P, const double* __restrict__ m, int64_t Ntot, int Lx,
                                           int Ly, int x, int y, int64_t layer, double3& b,
                                           std::integer_sequence<int, Kk...>) {
    (pair_term<S, Kk>(P, m, Ntot, Lx, Ly, x, y, layer, b), ...);
}

// pair field P_i = sum_o W_o m_{i+o} (no on-site term) of a lattice whose site 0
// is packed at `m` (SoA with component stride Ntot).  S = void: the plan's
// runtime offsets; S a compile-time shape (mj_shapes.hpp, in-layer offsets):
// its offsets unrolled, isotropic shells as one scalar each.
template <class S>
__device__ __forceinline__ double3 pair_field(const StencilParams& P, const double* __restrict__ m, int64_t Ntot,
                                              int Lx, int Ly, int Lz, int x, int y, int z) {
    double3 b = make_double3(0.0, 0.0, 0.0);
    if constexpr (std::is_void<S>::value) {
        for (int k = 0; k < P.n_off; ++k) {
            int64_t j;
            if (!neighbour_in(P, Lx, Ly, Lz, x, y, z, k, j)) continue;
            b = mat3(P.W[k], ld3(m, j, Ntot), b);
        }
    } else {
        pair_terms<S>(P, m, Ntot, Lx, Ly, x, y, static_cast<int64_t>(Lx) * Ly * z, b,
                      std::make_integer_sequence<int, S::K>{});
    }
    return b;
}

__device__ __forceinline__ double onsite_energy(const StencilParams& P, double3 s) {
    if (!P.has_onsite) return 0.0;
    return -0.5 * dot(s, mat3(P.W0, s, make_double3(0.0, 0.0, 0.0)));
}

// the proposal of a move (track_value.f90 sample_*); B the site's effective field
// -dE/dm (relaxationtype.f90 under- and over-relaxation)
__device__ __forceinline__ double3 propose(int proposal, double3 s, double3 B, double cos_cone, const uint32_t c[4],
                                           const double* __restrict__ tab) {
    if (proposal == MJ_MC_ISING) return make_double3(-s.x, -s.y, -s.z);
    if (proposal == MJ_MC_CONE) return cone_proposal(s, cos_cone, u32_open(c[0]), c[1], tab);
    const double sb = dot(s, B);
    double3 n;
    if (proposal == MJ_MC_UNDERRELAX) n = make_double3(s.x * (1.0 - sb) + B.x, s.y * (1.0 - sb) + B.y, s.z * (1.0 - sb) + B.z);
    else n = make_double3(B.x - s.x * (1.0 + sb), B.y - s.y * (1.0 + sb), B.z - s.z * (1.0 + sb));
    const double inv_n = 1.0 / sqrt(dot(n, n));
    return make_double3(n.x * inv_n, n.y * inv_n, n.z * inv_n);
}

// One Metropolis move of the site holding s (pair field Pf, Zeeman field zb):
// true and sn the new direction when taken, dE its energy change.  `site` is the
// index of the site within its lattice, the first word of the Philox counter;
// inv_kT = 1/kT.
__device__ __forceinline__ bool mc_move(const StencilParams& P, const uint32_t* keys, const double* __restrict__ tab,
                                        int proposal, double kT, double inv_kT, double cos_cone, uint32_t site,
                                        uint32_t sweep, uint32_t stream, double3 s, double3 Pf, double3 zb,
                                        double3& sn, double& dE) {
    uint32_t c[4] = {site, sweep, stream, kMcTag};
    philox10k(c, keys);
    double3 B = add3(Pf, zb);
    if (P.has_onsite) B = mat3(P.W0, s, B);
    sn = propose(proposal, s, B, cos_cone, c, tab);
    const double3 d = make_double3(sn.x - s.x, sn.y - s.y, sn.z - s.z);
    dE = -dot(d, Pf) + (onsite_energy(P, sn) - onsite_energy(P, s)) - dot(d, zb);
    bool acc = dE < 0.0;
    if (!acc && kT > 0.0) acc = u32_open(c[2]) < exp(fmax(-dE * inv_kT, -200.0));
    return acc;
}

// Colour-pass blocks of 32 x kMcBY threads: at 52-56 registers a thread, nine
// blocks of 128 threads fit an SM (36 warps) where blocks of 256 held four
// (32 warps).
constexpr int kMcBY = 4;

// One colour class of a sweep: the sites y = ry + sy ty, z = rz + sz tz,
// x = ((k - b y - c z) mod qx) + qx tx.  A linear colouring (q, b, c) has
// qx = q, sy = sz = 1, colour k; a product colouring (cx, cy, cz) has qx = cx,
// sy = cy, sz = cz, b = c = 0 and colour (k, ry, rz).
struct McClass {
    int qx, sy, sz, b, c, k, ry, rz;
};

__device__ __forceinline__ int mc_class_x(const McClass& K, int y, int z, int t) {
    return ((K.k - K.b * y - K.c * z) % K.qx + K.qx) % K.qx + K.qx * t;
}

// The colouring with the fewest colours (at least 2) in which no stencil offset
// joins two sites of one colour, on every lattice of sizes L[3 l .. 3 l + 2]:
// out = {q, b, c, 1} for the linear colour (x + b y + c z) mod q, or {cx, cy,
// cz, 0} for the product colour (x mod cx, y mod cy, z mod cz).  A periodic
// direction must map its wrapped images to the same colour (q divides every
// Lx, q divides b Ly and c Lz; cx divides every Lx, ...), so along a periodic
// direction the counts are the divisors of the sizes' greatest common divisor
// (a prime size p gives p colours), along an open one 2 .. 64.  Linear
// colourings up to 4096 colours, product ones up to 4096 in all.
inline bool mc_colouring(const StencilParams& sp, const int* L, int nlat, int out[4]) {
    auto gcd = [](int a, int b) {
        while (b) {
            const int t = a % b;
            a = b;
            b = t;
        }
        return a;
    };
    // counts allowed along direction d (ascending), from `lo`
    auto counts = [&](int d, int lo, int open_max) {
        std::vector<int> v;
        if (sp.periodic[d]) {
            int g = 0;
            for (int l = 0; l < nlat; ++l) g = gcd(g, L[3 * l + d]);
            for (int q = lo; q <= g; ++q)
                if (g % q == 0) v.push_back(q);
        } else {
            for (int q = lo; q <= open_max; ++q) v.push_back(q);
        }
        return v;
    };
    auto wraps_ok = [&](int d, int mult, int q) {
        if (!sp.periodic[d]) return true;
        for (int l = 0; l < nlat; ++l)
            if ((static_cast<int64_t>(mult) * L[3 * l + d]) % q) return false;
        return true;
    };
    bool zoff = false;  // any offset along z
    for (int k = 0; k < sp.n_off; ++k) zoff = zoff || sp.off[k][2] != 0;
    int best = 1 << 30;
    for (int q : counts(0, 2, 64)) {
        if (q >= best || q > 4096) break;
        const int cmax = zoff ? q : 1;  // without z offsets c = 0 serves every lattice
        for (int c = 0; c < cmax && q < best; ++c)
            for (int b = 0; b < q && q < best; ++b) {
                bool ok = wraps_ok(1, b, q) && wraps_ok(2, c, q);
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
    }
    const std::vector<int> cxs = counts(0, 1, 8), cys = counts(1, 1, 8), czs = counts(2, 1, 8);
    for (int cz : czs)
        for (int cy : cys)
            for (int cx : cxs) {
                const int64_t n = static_cast<int64_t>(cx) * cy * cz;
                if (n >= best || n <= 1 || n > 4096) continue;
                const int cc[3] = {cx, cy, cz};
                bool ok = true;
                for (int k = 0; k < sp.n_off && ok; ++k) {
                    bool differs = false;
                    for (int d = 0; d < 3; ++d) differs = differs || (((sp.off[k][d] % cc[d]) + cc[d]) % cc[d]) != 0;
                    ok = differs;
                }
                if (ok) {
                    best = static_cast<int>(n);
                    out[0] = cx;
                    out[1] = cy;
                    out[2] = cz;
                    out[3] = 0;
                }
            }
    return best < (1 << 30);
}

// the colour classes of a colouring in launch order
inline std::vector<McClass> mc_classes(const int col[4]) {
    std::vector<McClass> classes;
    if (col[3] == 1) {
        for (int k = 0; k < col[0]; ++k) classes.push_back({col[0], 1, 1, col[1], col[2], k, 0, 0});
    } else {
        for (int rz = 0; rz < col[2]; ++rz)
            for (int ry = 0; ry < col[1]; ++ry)
                for (int rx = 0; rx < col[0]; ++rx) classes.push_back({col[0], col[1], col[2], 0, 0, rx, ry, rz});
    }
    return classes;
}

// Philox4x32 round keys of a 64-bit seed (Weyl increments)
inline void mc_keys(uint64_t seed, uint32_t keys[20]) {
    uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        keys[2 * r] = k0;
        keys[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

}  // namespace
}  // namespace mj
