// One-site-per-thread access to a single-atom stencil plan: periodic
// neighbours, the real-space operator W (all coupling terms; the field is
// W m + Zeeman), the Zeeman field.  Shared by the reverse-mode and the
// minimisation kernels.
#pragma once

#include "mj_device.cuh"
#include "mj_internal.hpp"

namespace mj {
namespace {

// periodic image of a coordinate one offset away (one add in the common case)
__device__ __forceinline__ int wrap(int v, int L) {
    if (v < 0) {
        v += L;
        if (v < 0) v = ((v % L) + L) % L;
    } else if (v >= L) {
        v -= L;
        if (v >= L) v %= L;
    }
    return v;
}

__device__ __forceinline__ bool neighbour(const StencilParams& P, int x, int y, int z, int k, int64_t& j) {
    int nx = x + P.off[k][0], ny = y + P.off[k][1], nz = z + P.off[k][2];
    const int Lx = P.L[0], Ly = P.L[1], Lz = P.L[2];
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

__device__ __forceinline__ double3 mat3(const double* W, double3 v, double3 acc) {
    return make_double3(fma(W[0], v.x, fma(W[1], v.y, fma(W[2], v.z, acc.x))),
                        fma(W[3], v.x, fma(W[4], v.y, fma(W[5], v.z, acc.y))),
                        fma(W[6], v.x, fma(W[7], v.y, fma(W[8], v.z, acc.z))));
}
__device__ __forceinline__ double3 add3(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 scl3(double s, double3 a) { return make_double3(s * a.x, s * a.y, s * a.z); }

// (W v)_i of the real-space terms (no Zeeman)
__device__ __forceinline__ double3 w_apply(const StencilParams& P, const double* __restrict__ v, int64_t N, int x,
                                           int y, int z, double3 v0) {
    double3 b = make_double3(0.0, 0.0, 0.0);
    for (int k = 0; k < P.n_off; ++k) {
        int64_t j;
        if (!neighbour(P, x, y, z, k, j)) continue;
        const double3 a = ld3(v, j, N);
        if (P.iso[k]) {
            const double w = P.W[k][0];
            b = make_double3(fma(w, a.x, b.x), fma(w, a.y, b.y), fma(w, a.z, b.z));
        } else {
            b = mat3(P.W[k], a, b);
        }
    }
    if (P.has_onsite) b = mat3(P.W0, v0, b);
    return b;
}

__device__ __forceinline__ double3 zeeman(const StencilParams& P, const double* __restrict__ bmap, int64_t i,
                                          int64_t N) {
    if (!P.zee_on) return make_double3(0.0, 0.0, 0.0);
    double3 b;
    if (bmap) b = ld3(bmap, i, N);
    else b = make_double3(P.bext[0], P.bext[1], P.bext[2]);
    return scl3(P.zc, b);
}

}  // namespace
}  // namespace mj
