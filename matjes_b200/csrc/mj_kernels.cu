// Fused field + LLG kernels for the Matjes hot path (sm_100a, FP64).
//
// Every pass reads the spin field once (SoA, coalesced along x), evaluates the
// effective field of all real-space terms, and fuses the LLG torque and the
// integrator update into the same pass:
//   Euler        1 pass   : m' = P(m + (D + DT) h/hbar)            (solvers/solver.f90:97-118)
//   Heun-Matjes  2 passes : predictor m~, corrector from m~         (dynamics/spindynamics.f90:282-313)
//   SIB          2 passes : Cayley predictor -> midpoint, corrector (Mentink et al. 2010)
// The total energy of the incoming state (dynamics/spindynamics.f90:323) is
// reduced in the first pass at no extra DRAM traffic, deterministically
// (per-block partials summed in block order by the last block to finish).
//
// The passes are templates over a field provider: StencilField (single-atom
// cells; neighbour offsets and 3x3 tensors in the launch parameters) or
// EllField (multi-atom cells and COO input; per-site tensor lists).
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "mj_device.cuh"
#include "mj_internal.hpp"

namespace mj {
namespace {

// ---------------------------------------------------------------------------
// Field providers
struct StencilField {
    StencilParams P;
    const double* bmap;  // per-cell applied field, SoA (null = uniform)

    static constexpr int BX = 32, BY = 8;
    __device__ __forceinline__ int64_t nsites() const { return static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2]; }
    __device__ __forceinline__ bool site(int64_t& i, int& x, int& y, int& z) const {
        x = blockIdx.x * BX + threadIdx.x;
        y = blockIdx.y * BY + threadIdx.y;
        z = blockIdx.z;
        const bool a = x < P.L[0] && y < P.L[1];
        i = a ? x + static_cast<int64_t>(P.L[0]) * (y + static_cast<int64_t>(P.L[1]) * z) : 0;
        return a;
    }
    __device__ __forceinline__ FieldOut field(const double* __restrict__ m, int64_t i, int x, int y, int z, double3 m0) const {
        const int64_t N = nsites();
        const double* __restrict__ mx = m;
        const double* __restrict__ my = m + N;
        const double* __restrict__ mz = m + 2 * N;
        double bx = 0.0, by = 0.0, bz = 0.0;
        const int Lx = P.L[0], Ly = P.L[1], Lz = P.L[2];
        for (int k = 0; k < P.n_off; ++k) {
            int nx = x + P.off[k][0], ny = y + P.off[k][1], nz = z + P.off[k][2];
            if (nx < 0 || nx >= Lx) {
                if (!P.periodic[0]) continue;
                nx = ((nx % Lx) + Lx) % Lx;
            }
            if (ny < 0 || ny >= Ly) {
                if (!P.periodic[1]) continue;
                ny = ((ny % Ly) + Ly) % Ly;
            }
            if (nz < 0 || nz >= Lz) {
                if (!P.periodic[2]) continue;
                nz = ((nz % Lz) + Lz) % Lz;
            }
            const int64_t j = nx + static_cast<int64_t>(Lx) * (ny + static_cast<int64_t>(Ly) * nz);
            const double ax = __ldg(mx + j), ay = __ldg(my + j), az = __ldg(mz + j);
            const double* W = P.W[k];
            if (P.iso[k]) {
                const double w = W[0];
                bx = fma(w, ax, bx);
                by = fma(w, ay, by);
                bz = fma(w, az, bz);
            } else {
                bx = fma(W[0], ax, fma(W[1], ay, fma(W[2], az, bx)));
                by = fma(W[3], ax, fma(W[4], ay, fma(W[5], az, by)));
                bz = fma(W[6], ax, fma(W[7], ay, fma(W[8], az, bz)));
            }
        }
        if (P.has_onsite) {
            const double* W = P.W0;
            bx = fma(W[0], m0.x, fma(W[1], m0.y, fma(W[2], m0.z, bx)));
            by = fma(W[3], m0.x, fma(W[4], m0.y, fma(W[5], m0.z, by)));
            bz = fma(W[6], m0.x, fma(W[7], m0.y, fma(W[8], m0.z, bz)));
        }
        FieldOut f;
        f.Bzee = make_double3(0.0, 0.0, 0.0);
        if (P.zee_on) {
            double3 b;
            if (bmap) b = make_double3(__ldg(bmap + i), __ldg(bmap + N + i), __ldg(bmap + 2 * N + i));
            else b = make_double3(P.bext[0], P.bext[1], P.bext[2]);
            f.Bzee = make_double3(P.zc * b.x, P.zc * b.y, P.zc * b.z);
        }
        f.B = make_double3(bx + f.Bzee.x, by + f.Bzee.y, bz + f.Bzee.z);
        return f;
    }
};

struct EllField {
    int64_t N;
    int64_t ncell;
    int nmag;
    int width;
    const int* col;      // [width][N]
    const double* val;   // [width][9][N]
    const double* zc;    // [N]
    const double* bmap;  // per-cell SoA (null = uniform bext)
    double bext[3];
    int zee_on;

    static constexpr int BX = 256, BY = 1;
    __device__ __forceinline__ int64_t nsites() const { return N; }
    __device__ __forceinline__ bool site(int64_t& i, int& x, int& y, int& z) const {
        i = blockIdx.x * static_cast<int64_t>(BX) + threadIdx.x;
        x = y = z = 0;
        const bool a = i < N;
        if (!a) i = 0;
        return a;
    }
    __device__ __forceinline__ FieldOut field(const double* __restrict__ m, int64_t i, int, int, int, double3) const {
        double bx = 0.0, by = 0.0, bz = 0.0;
        for (int k = 0; k < width; ++k) {
            const int j = __ldg(col + static_cast<int64_t>(k) * N + i);
            if (j < 0) continue;
            const double ax = __ldg(m + j), ay = __ldg(m + N + j), az = __ldg(m + 2 * N + j);
            const double* W = val + static_cast<int64_t>(k) * 9 * N + i;
            bx = fma(__ldg(W + 0 * N), ax, fma(__ldg(W + 1 * N), ay, fma(__ldg(W + 2 * N), az, bx)));
            by = fma(__ldg(W + 3 * N), ax, fma(__ldg(W + 4 * N), ay, fma(__ldg(W + 5 * N), az, by)));
            bz = fma(__ldg(W + 6 * N), ax, fma(__ldg(W + 7 * N), ay, fma(__ldg(W + 8 * N), az, bz)));
        }
        FieldOut f;
        f.Bzee = make_double3(0.0, 0.0, 0.0);
        if (zee_on) {
            const int64_t c = i / nmag;
            double3 b;
            if (bmap) b = make_double3(__ldg(bmap + c), __ldg(bmap + ncell + c), __ldg(bmap + 2 * ncell + c));
            else b = make_double3(bext[0], bext[1], bext[2]);
            const double z = __ldg(zc + i);
            f.Bzee = make_double3(z * b.x, z * b.y, z * b.z);
        }
        f.B = make_double3(bx + f.Bzee.x, by + f.Bzee.y, bz + f.Bzee.z);
        return f;
    }
};

struct Reduce {
    double* partials;
    unsigned int* counter;
    double* out;  // null = no energy wanted
    int nblocks;
};

__device__ __forceinline__ double3 minus2(double3 B, double3 hd) {
    return make_double3(B.x - 2.0 * hd.x, B.y - 2.0 * hd.y, B.z - 2.0 * hd.z);
}

// ---------------------------------------------------------------------------
template <class F>
__global__ void __launch_bounds__(256) k_field(const __grid_constant__ F fp, const double* __restrict__ m,
                                               const DipView Hd, double* __restrict__ B,
                                               double* __restrict__ e_site, Reduce R) {
    int64_t i;
    int x, y, z;
    const bool act = fp.site(i, x, y, z);
    const int64_t N = fp.nsites();
    double e = 0.0;
    if (act) {
        const double3 m0 = ld3(m, i, N);
        const FieldOut f = fp.field(m, i, x, y, z, m0);
        const double3 hd = Hd.h ? ld_dip(Hd, x, y, z) : make_double3(0.0, 0.0, 0.0);
        if (B) st3(B, i, N, minus2(f.B, hd));
        if (e_site) e_site[i] = site_energy(f, m0, hd);
        e = total_energy_part(f, m0, hd);
    }
    if (R.out) {
        double v[1] = {e};
        grid_reduce<1>(v, R.partials, R.counter, R.out, R.nblocks);
    }
}

// Euler: one fused pass m -> mout.
template <class F>
__global__ void __launch_bounds__(256) k_euler(const __grid_constant__ F fp, const DynCoef C, uint32_t step,
                                               const double* __restrict__ m, double* __restrict__ mout,
                                               const DipView Hd, Reduce R, int* status, const DipPad pad) {
    int64_t i;
    int x, y, z;
    const bool act = fp.site(i, x, y, z);
    const int64_t N = fp.nsites();
    double e = 0.0;
    if (act) {
        const double3 m0 = ld3(m, i, N);
        const FieldOut f = fp.field(m, i, x, y, z, m0);
        const double3 hd = Hd.h ? ld_dip(Hd, x, y, z) : make_double3(0.0, 0.0, 0.0);
        e = total_energy_part(f, m0, hd);
        const double3 D = llg_rhs(minus2(f.B, hd), m0, C.alpha, C.inv_den);
        const double c = C.h_over_hbar;
        double3 t = make_double3(m0.x + D.x * c, m0.y + D.y * c, m0.z + D.z * c);
        if (C.thermal) {
            const double3 DT = llg_rhs(thermal_field(C, step, i, N), m0, C.alpha, C.inv_den);
            t = make_double3(t.x + DT.x * c, t.y + DT.y * c, t.z + DT.z * c);
        }
        const double3 mo = project(t, m0);
        flag_nonfinite(status, mo);
        st3(mout, i, N, mo);
        if (pad.p) st_pad(pad, x, y, z, mo);
    }
    if (R.out) {
        double v[1] = {e};
        grid_reduce<1>(v, R.partials, R.counter, R.out, R.nblocks);
    }
}

// Heun-Matjes pass 1: predictor m~ = P(m + D1 h/hbar); keeps D1 and DT for pass 2.
template <class F>
__global__ void __launch_bounds__(256) k_heun1(const __grid_constant__ F fp, const DynCoef C, uint32_t step,
                                               const double* __restrict__ m, double* __restrict__ mid,
                                               double* __restrict__ D1, double* __restrict__ DTo,
                                               const DipView Hd, Reduce R, const DipPad pad) {
    int64_t i;
    int x, y, z;
    const bool act = fp.site(i, x, y, z);
    const int64_t N = fp.nsites();
    double e = 0.0;
    if (act) {
        const double3 m0 = ld3(m, i, N);
        const FieldOut f = fp.field(m, i, x, y, z, m0);
        const double3 hd = Hd.h ? ld_dip(Hd, x, y, z) : make_double3(0.0, 0.0, 0.0);
        e = total_energy_part(f, m0, hd);
        const double3 D = llg_rhs(minus2(f.B, hd), m0, C.alpha, C.inv_den);
        const double c = C.h_over_hbar;
        const double3 t = make_double3(m0.x + D.x * c, m0.y + D.y * c, m0.z + D.z * c);
        const double3 mt = project(t, m0);
        st3(mid, i, N, mt);
        if (pad.p) st_pad(pad, x, y, z, mt);
        st3(D1, i, N, D);
        if (C.thermal) st3(DTo, i, N, llg_rhs(thermal_field(C, step, i, N), m0, C.alpha, C.inv_den));
    }
    if (R.out) {
        double v[1] = {e};
        grid_reduce<1>(v, R.partials, R.counter, R.out, R.nblocks);
    }
}

// Heun-Matjes pass 2: corrector restarted from the predictor.
template <class F>
__global__ void __launch_bounds__(256) k_heun2(const __grid_constant__ F fp, const DynCoef C,
                                               const double* __restrict__ mid, const double* __restrict__ D1,
                                               const double* __restrict__ DTi, double* __restrict__ mout,
                                               const DipView Hd, int* status, const DipPad pad) {
    int64_t i;
    int x, y, z;
    if (!fp.site(i, x, y, z)) return;
    const int64_t N = fp.nsites();
    const double3 mt = ld3(mid, i, N);
    const FieldOut f = fp.field(mid, i, x, y, z, mt);
    const double3 hd = Hd.h ? ld_dip(Hd, x, y, z) : make_double3(0.0, 0.0, 0.0);
    const double3 D2 = llg_rhs(minus2(f.B, hd), mt, C.alpha, C.inv_den);
    const double3 d1 = ld3(D1, i, N);
    const double3 Di = make_double3(0.5 * d1.x + 0.5 * D2.x, 0.5 * d1.y + 0.5 * D2.y, 0.5 * d1.z + 0.5 * D2.z);
    const double c = C.h_over_hbar;
    double3 t = make_double3(mt.x + Di.x * c, mt.y + Di.y * c, mt.z + Di.z * c);
    if (C.thermal) {
        const double3 DT = ld3(DTi, i, N);
        t = make_double3(t.x + DT.x * c, t.y + DT.y * c, t.z + DT.z * c);
    }
    const double3 mo = project(t, mt);
    flag_nonfinite(status, mo);
    st3(mout, i, N, mo);
    if (pad.p) st_pad(pad, x, y, z, mo);
}

// SIB pass 1: Cayley predictor from m_n with A(m_n); writes the midpoint (m_n + m~)/2.
template <class F>
__global__ void __launch_bounds__(256) k_sib1(const __grid_constant__ F fp, const DynCoef C, uint32_t step,
                                              const double* __restrict__ m, double* __restrict__ mid,
                                              const DipView Hd, Reduce R, const DipPad pad) {
    int64_t i;
    int x, y, z;
    const bool act = fp.site(i, x, y, z);
    const int64_t N = fp.nsites();
    double e = 0.0;
    if (act) {
        const double3 m0 = ld3(m, i, N);
        const FieldOut f = fp.field(m, i, x, y, z, m0);
        const double3 hd = Hd.h ? ld_dip(Hd, x, y, z) : make_double3(0.0, 0.0, 0.0);
        e = total_energy_part(f, m0, hd);
        double3 H = minus2(f.B, hd);
        if (C.thermal) {
            const double3 b = thermal_field(C, step, i, N);
            H = make_double3(H.x + b.x, H.y + b.y, H.z + b.z);
        }
        const double3 mb = sib_solve<true>(m0, m0, H, C.alpha, C.sib_hc);
        st3(mid, i, N, mb);
        if (pad.p) st_pad(pad, x, y, z, mb);
    }
    if (R.out) {
        double v[1] = {e};
        grid_reduce<1>(v, R.partials, R.counter, R.out, R.nblocks);
    }
}

// SIB pass 2: corrector from m_n with A(midpoint); in place (only the own site of m is read).
template <class F>
__global__ void __launch_bounds__(256) k_sib2(const __grid_constant__ F fp, const DynCoef C, uint32_t step,
                                              const double* __restrict__ mid, double* m, const DipView Hd,
                                              int* status, const DipPad pad) {
    int64_t i;
    int x, y, z;
    if (!fp.site(i, x, y, z)) return;
    const int64_t N = fp.nsites();
    const double3 mb = ld3(mid, i, N);
    const FieldOut f = fp.field(mid, i, x, y, z, mb);
    const double3 hd = Hd.h ? ld_dip(Hd, x, y, z) : make_double3(0.0, 0.0, 0.0);
    double3 H = minus2(f.B, hd);
    if (C.thermal) {
        const double3 b = thermal_field(C, step, i, N);
        H = make_double3(H.x + b.x, H.y + b.y, H.z + b.z);
    }
    const double3 m0 = make_double3(m[i], m[N + i], m[2 * N + i]);
    const double3 mo = sib_solve(m0, mb, H, C.alpha, C.sib_hc);
    flag_nonfinite(status, mo);
    st3(m, i, N, mo);
    if (pad.p) st_pad(pad, x, y, z, mo);
}

// Reference temperature estimator (dynamics/measure_temp.f90:21-43): sum |m x B|^2, sum m.B.
template <class F>
__global__ void __launch_bounds__(256) k_temperature(const __grid_constant__ F fp, const double* __restrict__ m,
                                                     const DipView Hd, Reduce R) {
    int64_t i;
    int x, y, z;
    const bool act = fp.site(i, x, y, z);
    const int64_t N = fp.nsites();
    double v[2] = {0.0, 0.0};
    if (act) {
        const double3 m0 = ld3(m, i, N);
        const FieldOut f = fp.field(m, i, x, y, z, m0);
        const double3 hd = Hd.h ? ld_dip(Hd, x, y, z) : make_double3(0.0, 0.0, 0.0);
        const double3 Bt = minus2(f.B, hd);
        const double3 c = cross(m0, Bt);
        v[0] = dot(c, c);
        v[1] = dot(m0, Bt);
    }
    grid_reduce<2>(v, R.partials, R.counter, R.out, R.nblocks);
}

__global__ void k_philox(uint64_t seed, uint32_t step, uint32_t stream, int64_t n, double* out, const double* tab) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double3 z = philox_normals(seed, step, stream, static_cast<uint32_t>(i), tab);
    out[i] = z.x;
    out[n + i] = z.y;
    out[2 * n + i] = z.z;
}

__global__ void k_step_counter(uint32_t* ctr, uint32_t value, int add) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *ctr = add ? *ctr + value : value;
}

__global__ void k_aos_to_soa(const double* __restrict__ a, double* __restrict__ s, int64_t n) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    s[i] = a[3 * i];
    s[n + i] = a[3 * i + 1];
    s[2 * n + i] = a[3 * i + 2];
}
// the same transposes over the sites [i0, i0 + cnt) of n
__global__ void k_aos_to_soa_range(const double* __restrict__ a, double* __restrict__ s, int64_t i0, int64_t cnt,
                                   int64_t n) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= cnt) return;
    const int64_t i = i0 + t;
    s[i] = a[3 * i];
    s[n + i] = a[3 * i + 1];
    s[2 * n + i] = a[3 * i + 2];
}
__global__ void k_soa_to_aos_range(const double* __restrict__ s, double* __restrict__ a, int64_t i0, int64_t cnt,
                                   int64_t n) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= cnt) return;
    const int64_t i = i0 + t;
    a[3 * i] = s[i];
    a[3 * i + 1] = s[n + i];
    a[3 * i + 2] = s[2 * n + i];
}
// The same into memory across the host link (a mapped pinned host buffer): a
// block's 256 sites staged in shared memory as AoS, then written contiguously
// (consecutive threads on consecutive addresses), 16 bytes a thread where the
// block's span starts on a 16-byte boundary, else 8.
__global__ void __launch_bounds__(256) k_soa_to_aos_stream(const double* __restrict__ s, double* __restrict__ a,
                                                           int64_t i0, int64_t cnt, int64_t n) {
    __shared__ __align__(16) double buf[3 * 256];
    const int64_t base = i0 + blockIdx.x * static_cast<int64_t>(256);
    const int64_t end = i0 + cnt;
    const int t = threadIdx.x;
    const int64_t i = base + t;
    if (i < end) {
        buf[3 * t] = s[i];
        buf[3 * t + 1] = s[n + i];
        buf[3 * t + 2] = s[2 * n + i];
    }
    __syncthreads();
    const int nd = 3 * static_cast<int>(end - base < 256 ? end - base : 256);
    double* dst = a + 3 * base;
    if ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
        const int np = nd / 2;  // whole 16-byte pairs, then an odd last double
        double2* d2 = reinterpret_cast<double2*>(dst);
        const double2* b2 = reinterpret_cast<const double2*>(buf);
        for (int k = t; k < np; k += 256) d2[k] = b2[k];
        if ((nd & 1) && t == 0) dst[nd - 1] = buf[nd - 1];
    } else {
        for (int k = t; k < nd; k += 256) dst[k] = buf[k];
    }
}
// energy partials summed in the fixed order of ordered_sum (one block)
__global__ void k_ordered_sum1(const double* partials, int nblocks, double* out) { ordered_sum<1>(partials, nblocks, out); }

__global__ void k_soa_to_aos(const double* __restrict__ s, double* __restrict__ a, int64_t n) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    a[3 * i] = s[i];
    a[3 * i + 1] = s[n + i];
    a[3 * i + 2] = s[2 * n + i];
}

// ---------------------------------------------------------------------------
StencilField stencil_of(const mj_plan* p) {
    StencilField f;
    f.P = p->sp;
    f.bmap = p->d_bmap;
    return f;
}
EllField ell_of(const mj_plan* p) {
    EllField f;
    f.N = p->N;
    f.ncell = p->ncell;
    f.nmag = p->nmag;
    f.width = p->ell_width;
    f.col = p->d_ell_col;
    f.val = p->d_ell_val;
    f.zc = p->d_zee;
    f.bmap = p->d_bmap;
    for (int k = 0; k < 3; ++k) f.bext[k] = p->bext_cell.size() == 3 ? p->bext_cell[k] : 0.0;
    f.zee_on = p->d_zee != nullptr;
    return f;
}
dim3 grid_stencil(const StencilParams& P) {
    return dim3((P.L[0] + StencilField::BX - 1) / StencilField::BX, (P.L[1] + StencilField::BY - 1) / StencilField::BY, P.L[2]);
}
dim3 grid_ell(int64_t N) { return dim3(static_cast<unsigned>((N + EllField::BX - 1) / EllField::BX), 1, 1); }

template <class F>
struct Launch {
    F fp;
    dim3 grid, block;
};

Reduce make_reduce(mj_plan* p, double* out) {
    Reduce r;
    r.partials = p->d_partials;
    r.counter = p->d_counter;
    r.out = out;
    r.nblocks = static_cast<int>(energy_blocks(p));
    return r;
}

DipView dip_field(mj_plan* p, const double* m, cudaStream_t s, mj_status& st) {
    st = MJ_OK;
    if (p->dip_on) {
        const int r = prof_begin(p, "dipolar_fft", s);
        st = dipolar_apply(p, m, nullptr, s);
        prof_end(p, r, s);
    }
    return dipolar_view(p);
}

#define MJ_LAUNCH(name, kern, ...)                                  \
    do {                                                            \
        const int rec_ = prof_begin(p, name, s);                    \
        kern<<<L.grid, L.block, 0, s>>>(__VA_ARGS__);               \
        prof_end(p, rec_, s);                                       \
        if ((st = cuda_status(cudaGetLastError(), name)) != MJ_OK) return st; \
    } while (0)

template <class F>
mj_status field_impl(mj_plan* p, const Launch<F>& L, const double* m, double* B, double* e_site, double* E_out,
                     cudaStream_t s) {
    mj_status st;
    DipView Hd = dip_field(p, m, s, st);
    if (st != MJ_OK) return st;
    MJ_LAUNCH("k_field", k_field<F>, L.fp, m, Hd, B, e_site, make_reduce(p, E_out));
    return MJ_OK;
}

// One time step.  Euler writes m_out (ping-pong owned by the caller); the
// two-pass schemes update m in place through the plan's midpoint buffer.
template <class F>
mj_status step_impl(mj_plan* p, const Launch<F>& L, double* m, double* m_out, const DynCoef& c, uint32_t step,
                    double* E_prev, cudaStream_t s) {
    mj_status st;
    // inside a step sequence with the dipolar term: every pass also writes its
    // spins into the padded grid of the next dipolar evaluation
    const DipPad pd = (p->dip_on && p->dip_fuse_pad) ? dipolar_pad(p) : DipPad{nullptr, 0, 0, 0};
    switch (c.integrator) {
        case MJ_EULER: {
            DipView Hd = dip_field(p, m, s, st);
            if (st != MJ_OK) return st;
            MJ_LAUNCH("k_euler", k_euler<F>, L.fp, c, step, m, m_out, Hd, make_reduce(p, E_prev), p->d_status, pd);
            if (pd.p) p->dip_pad_holds = m_out;
            return MJ_OK;
        }
        case MJ_HEUN_MATJES: {
            DipView Hd = dip_field(p, m, s, st);
            if (st != MJ_OK) return st;
            MJ_LAUNCH("k_heun1", k_heun1<F>, L.fp, c, step, m, p->d_mid, p->d_aux, p->d_aux2, Hd, make_reduce(p, E_prev),
                      pd);
            if (pd.p) p->dip_pad_holds = p->d_mid;
            Hd = dip_field(p, p->d_mid, s, st);
            if (st != MJ_OK) return st;
            MJ_LAUNCH("k_heun2", k_heun2<F>, L.fp, c, p->d_mid, p->d_aux, p->d_aux2, m, Hd, p->d_status, pd);
            if (pd.p) p->dip_pad_holds = m;
            return MJ_OK;
        }
        case MJ_SIB: {
            DipView Hd = dip_field(p, m, s, st);
            if (st != MJ_OK) return st;
            MJ_LAUNCH("k_sib1", k_sib1<F>, L.fp, c, step, m, p->d_mid, Hd, make_reduce(p, E_prev), pd);
            if (pd.p) p->dip_pad_holds = p->d_mid;
            Hd = dip_field(p, p->d_mid, s, st);
            if (st != MJ_OK) return st;
            MJ_LAUNCH("k_sib2", k_sib2<F>, L.fp, c, step, p->d_mid, m, Hd, p->d_status, pd);
            if (pd.p) p->dip_pad_holds = m;
            return MJ_OK;
        }
        default:
            return set_error(MJ_ERR_ARG, "unknown integrator");
    }
}

template <class F>
mj_status temperature_impl(mj_plan* p, const Launch<F>& L, const double* m, double* out2, cudaStream_t s) {
    mj_status st;
    DipView Hd = dip_field(p, m, s, st);
    if (st != MJ_OK) return st;
    k_temperature<F><<<L.grid, L.block, 0, s>>>(L.fp, m, Hd, make_reduce(p, out2));
    return cuda_status(cudaGetLastError(), "k_temperature");
}

Launch<StencilField> stencil_launch(const mj_plan* p) {
    return Launch<StencilField>{stencil_of(p), grid_stencil(p->sp), dim3(StencilField::BX, StencilField::BY)};
}
Launch<EllField> ell_launch(const mj_plan* p) {
    return Launch<EllField>{ell_of(p), grid_ell(p->N), dim3(EllField::BX, 1)};
}

}  // namespace

int64_t energy_blocks(const mj_plan* p) {
    if (p->is_stencil) {
        const dim3 g = grid_stencil(p->sp);
        return static_cast<int64_t>(g.x) * g.y * g.z;
    }
    return grid_ell(p->N).x;
}

namespace {

bool tiled(const mj_plan* p) { return p->is_stencil && p->sp.shape != 0; }

mj_status tiled_call(mj_plan* p, const char* name, int pass, const DynCoef& c, const double* ms, const double* mn,
                     double* out, double* aux, double* aux2, DipView Hd, double* E, uint32_t step, cudaStream_t s,
                     int emode = 0) {
    const int rec = prof_begin(p, name, s);
    mj_status st = launch_tiled(p, pass, c, ms, mn, out, aux, aux2, Hd, E, step, s, emode);
    prof_end(p, rec, s);
    return st;
}

mj_status tiled_field(mj_plan* p, const double* m, double* B, double* e_site, double* E_out, cudaStream_t s) {
    mj_status st;
    DipView Hd = dip_field(p, m, s, st);
    if (st != MJ_OK) return st;
    DynCoef c{};
    return tiled_call(p, "k_field", 0, c, m, nullptr, B, e_site, nullptr, Hd, E_out, 0u, s);
}

mj_status tiled_step(mj_plan* p, double* m, double* m_out, const DynCoef& c, uint32_t step, double* E_prev,
                     cudaStream_t s) {
    mj_status st;
    DipView Hd = dip_field(p, m, s, st);
    if (st != MJ_OK) return st;
    switch (c.integrator) {
        case MJ_EULER:
            return tiled_call(p, "k_euler", 1, c, m, nullptr, m_out, nullptr, nullptr, Hd, E_prev, step, s);
        // two-pass schemes: pass 1 writes per-block energy partials, the first block
        // of pass 2 sums them (no ticket or last-block tail in pass 1)
        case MJ_HEUN_MATJES:
            if ((st = tiled_call(p, "k_heun1", 2, c, m, nullptr, p->d_mid, p->d_aux, p->d_aux2, Hd, nullptr, step, s,
                                 E_prev ? 1 : 0)) != MJ_OK)
                return st;
            Hd = dip_field(p, p->d_mid, s, st);
            if (st != MJ_OK) return st;
            return tiled_call(p, "k_heun2", 3, c, p->d_mid, nullptr, m, p->d_aux, p->d_aux2, Hd, E_prev, step, s,
                              E_prev ? 2 : 0);
        case MJ_SIB: {
            // Philox draws are made once per step in pass 1 and kept for the corrector
            double* bstore = (c.thermal && c.noise == MJ_NOISE_PHILOX && p->store_draw) ? p->d_aux : nullptr;
            if (p->fused_sib && !p->dip_on && p->d_sched) {  // predictor and corrector in one launch
                const int rec = prof_begin(p, "k_sib_fused", s);
                st = launch_sib_fused(p, c, m, bstore, E_prev, step, s);
                prof_end(p, rec, s);
                return st;
            }
            if ((st = tiled_call(p, "k_sib1", 4, c, m, nullptr, p->d_mid, bstore, nullptr, Hd, nullptr, step, s,
                                 E_prev ? 1 : 0)) != MJ_OK)
                return st;
            Hd = dip_field(p, p->d_mid, s, st);
            if (st != MJ_OK) return st;
            return tiled_call(p, "k_sib2", 5, c, p->d_mid, m, m, bstore, nullptr, Hd, E_prev, step, s, E_prev ? 2 : 0);
        }
        default:
            return set_error(MJ_ERR_ARG, "unknown integrator");
    }
}

}  // namespace

mj_status launch_field(mj_plan* p, const double* m, double* B, double* e_site, double* E_out, cudaStream_t s) {
    if (tiled(p)) return tiled_field(p, m, B, e_site, E_out, s);
    if (p->is_stencil) return field_impl(p, stencil_launch(p), m, B, e_site, E_out, s);
    return field_impl(p, ell_launch(p), m, B, e_site, E_out, s);
}

mj_status launch_energy(mj_plan* p, const double* m, double* E_out, cudaStream_t s) {
    return launch_field(p, m, nullptr, nullptr, E_out, s);
}

mj_status launch_step(mj_plan* p, double* m, double* m_out, const DynCoef& c, uint32_t step, double* E_prev_out,
                      cudaStream_t s) {
    if (tiled(p)) return tiled_step(p, m, m_out, c, step, E_prev_out, s);
    if (p->is_stencil) return step_impl(p, stencil_launch(p), m, m_out, c, step, E_prev_out, s);
    return step_impl(p, ell_launch(p), m, m_out, c, step, E_prev_out, s);
}

mj_status launch_temperature(mj_plan* p, const double* m, double* out2, cudaStream_t s) {
    if (p->is_stencil) return temperature_impl(p, stencil_launch(p), m, out2, s);
    return temperature_impl(p, ell_launch(p), m, out2, s);
}

mj_status launch_philox(uint64_t seed, uint32_t step, uint32_t stream_id, int64_t n, double* out, cudaStream_t s) {
    if (n <= 0) return MJ_OK;
    // Box-Muller tables of the current device, built once per device
    static double* tabs[64] = {nullptr};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(MJ_ERR_ARG, "device index out of range");
    if (!tabs[dev]) {
        std::vector<double> h(kNoiseTabDoubles);
        build_noise_tables(h.data());
        const size_t bytes = sizeof(double) * kNoiseTabDoubles;
        mj_status st = cuda_status(cudaMalloc(&tabs[dev], bytes), "philox tables");
        if (st != MJ_OK) return st;
        if ((st = cuda_status(cudaMemcpy(tabs[dev], h.data(), bytes, cudaMemcpyHostToDevice), "philox tables")) != MJ_OK)
            return st;
    }
    k_philox<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(seed, step, stream_id, n, out, tabs[dev]);
    return cuda_status(cudaGetLastError(), "k_philox");
}

mj_status step_counter(uint32_t* ctr, uint32_t value, bool add, cudaStream_t s) {
    k_step_counter<<<1, 32, 0, s>>>(ctr, value, add ? 1 : 0);
    return cuda_status(cudaGetLastError(), "k_step_counter");
}

mj_status aos_to_soa(const double* a, double* so, int64_t n, cudaStream_t s) {
    if (n <= 0) return MJ_OK;
    k_aos_to_soa<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(a, so, n);
    return cuda_status(cudaGetLastError(), "aos_to_soa");
}
mj_status aos_to_soa_range(const double* a, double* so, int64_t i0, int64_t cnt, int64_t n, cudaStream_t s) {
    if (cnt <= 0) return MJ_OK;
    k_aos_to_soa_range<<<static_cast<unsigned>((cnt + 255) / 256), 256, 0, s>>>(a, so, i0, cnt, n);
    return cuda_status(cudaGetLastError(), "aos_to_soa_range");
}
mj_status soa_to_aos_range(const double* so, double* a, int64_t i0, int64_t cnt, int64_t n, cudaStream_t s) {
    if (cnt <= 0) return MJ_OK;
    k_soa_to_aos_range<<<static_cast<unsigned>((cnt + 255) / 256), 256, 0, s>>>(so, a, i0, cnt, n);
    return cuda_status(cudaGetLastError(), "soa_to_aos_range");
}
mj_status soa_to_aos_stream(const double* so, double* a, int64_t i0, int64_t cnt, int64_t n, cudaStream_t s) {
    if (cnt <= 0) return MJ_OK;
    k_soa_to_aos_stream<<<static_cast<unsigned>((cnt + 255) / 256), 256, 0, s>>>(so, a, i0, cnt, n);
    return cuda_status(cudaGetLastError(), "soa_to_aos_stream");
}
mj_status launch_ordered_sum(const double* partials, int nblocks, int nthreads, double* out, cudaStream_t s) {
    k_ordered_sum1<<<1, nthreads, 0, s>>>(partials, nblocks, out);
    return cuda_status(cudaGetLastError(), "k_ordered_sum1");
}
mj_status soa_to_aos(const double* so, double* a, int64_t n, cudaStream_t s) {
    if (n <= 0) return MJ_OK;
    k_soa_to_aos<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(so, a, n);
    return cuda_status(cudaGetLastError(), "soa_to_aos");
}

// ---------------------------------------------------------------------------
// Energy with no allocation (mj_energy_noalloc).  The reduction scratch is this
// fixed array: MJ_NOALLOC_MAX_BLOCKS per-block partial sums, then the ticket
// counter in the first 4 bytes of the slot after them.  Every GPU that loads
// the library holds it until exit; all calls on a device share it.
static __device__ __align__(256) double g_noalloc_scratch[MJ_NOALLOC_MAX_BLOCKS + 32];

namespace {

__global__ void k_noalloc_arm(unsigned int* counter) {
    if (threadIdx.x == 0) *counter = 0u;  // a previous call may have stopped before re-arming it
}

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array on the current device, looked up once per
// device (host code cannot use the symbol's name as a device pointer).
mj_status noalloc_scratch(double** out) {
    int dev = -1;
    mj_status st = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
    if (st != MJ_OK) return st;
    if (dev < 0 || dev >= 64) return set_error(MJ_ERR_ARG, "device index out of range for the no-allocation scratch");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        if ((st = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-allocation scratch)")) !=
            MJ_OK)
            return st;
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return MJ_OK;
}

}  // namespace

}  // namespace mj

extern "C" mj_status mj_energy_noalloc(const mj_plan* plan, const double* m, double* E, void* stream) {
    using namespace mj;
    if (!plan || !m || !E) return set_error(MJ_ERR_ARG, "null argument");
    if (plan->dip_on)
        return set_error(MJ_ERR_UNSUPPORTED, "the FFT dipolar term needs the plan's FFT buffers; use mj_energy");
    mj_status st = cuda_status(cudaSetDevice(plan->device), "cudaSetDevice");
    if (st != MJ_OK) return st;
    const int64_t nblocks = energy_blocks(plan);
    if (nblocks > MJ_NOALLOC_MAX_BLOCKS)
        return set_error(MJ_ERR_ARG, "lattice needs " + std::to_string(nblocks) +
                                         " thread blocks; the no-allocation scratch holds MJ_NOALLOC_MAX_BLOCKS = " +
                                         std::to_string(MJ_NOALLOC_MAX_BLOCKS) +
                                         " (one per 32 x 8 tile of a layer, or per 256 sites of an ELL plan)");
    double* scratch = nullptr;
    if ((st = noalloc_scratch(&scratch)) != MJ_OK) return st;
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + MJ_NOALLOC_MAX_BLOCKS);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_noalloc_arm<<<1, 32, 0, s>>>(counter);
    if ((st = cuda_status(cudaGetLastError(), "k_noalloc_arm")) != MJ_OK) return st;
    Reduce R;
    R.partials = scratch;
    R.counter = counter;
    R.out = E;
    R.nblocks = static_cast<int>(nblocks);
    DipView none;
    none.h = nullptr;
    none.cs = none.zs = 0;
    none.px = 0;
    if (plan->is_stencil) {
        const Launch<StencilField> L = stencil_launch(plan);
        k_field<StencilField><<<L.grid, L.block, 0, s>>>(L.fp, m, none, nullptr, nullptr, R);
    } else {
        const Launch<EllField> L = ell_launch(plan);
        k_field<EllField><<<L.grid, L.block, 0, s>>>(L.fp, m, none, nullptr, nullptr, R);
    }
    return cuda_status(cudaGetLastError(), "k_field (no allocation)");
}
