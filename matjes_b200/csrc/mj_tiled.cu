// Shared-memory tiled stencil passes for the lattices with compile-time offset
// tables (mj_shapes.hpp): square NN / NN+NNN, triangular NN / three shells.
//
// A block of 32 x BYT threads owns a 32 x (BYT*RY) tile of one z-layer; each
// thread owns RY sites stacked along y.  The tile plus its halo (radius R) is
// staged once in shared memory (SoA, periodic wrap or open-boundary zeros
// resolved at load time), then each thread walks the stencil column by column:
// a value of column dx is loaded once and accumulated into every one of the
// thread's RY sites that sees it, so a site costs ~(RY + span)/RY loads per
// column instead of one load per offset.  Offsets and tensor slots are
// compile-time constants; the coupling values come from the launch parameters.
// The integrator epilogues are the same device functions as the generic path.
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "mj_device.cuh"
#include "mj_internal.hpp"
#include "mj_shapes.hpp"

namespace mj {
namespace {

enum { PASS_FIELD = 0, PASS_EULER = 1, PASS_HEUN1 = 2, PASS_HEUN2 = 3, PASS_SIB1 = 4, PASS_SIB2 = 5 };

struct TReduce {
    double* partials;
    unsigned int* counter;
    double* out;
    int nblocks;
};

struct TiledArgs {
    const double* ms;   // spins the stencil runs on (m, or the midpoint in pass 2)
    const double* mn;   // m_n (own site) for the SIB corrector
    double* out;        // field B / next state / midpoint
    double* aux;        // Heun D1, or per-site energy for the field pass
    double* aux2;       // Heun DT
    const double* bmap; // per-cell applied field (SoA) or null
    DipView Hd;
    TReduce R;
    uint32_t step;
};

template <class S, int BYT, int RY>
struct TileGeom {
    static constexpr int R = S::R;
    static constexpr int TX = 32, TY = BYT * RY;
    static constexpr int PX = TX + 2 * R;
    static constexpr int PY = TY + 2 * R;
    static constexpr int NS = PX * PY;
    static constexpr size_t smem_bytes = sizeof(double) * 3 * NS;
};

// contribution of one loaded stencil row (column DX, row YY relative to the
// thread's first site) to the thread's RY accumulators
template <class S, int RY, int DX, int YY, int... Kk>
__device__ __forceinline__ void row_accumulate(const StencilParams& P, double vx, double vy, double vz, double* bx,
                                               double* by, double* bz, std::integer_sequence<int, Kk...>) {
    (
        [&] {
            constexpr int k = Kk;
            if constexpr (S::DX[k] == DX) {
                constexpr int r = YY - S::DY[k];
                if constexpr (r >= 0 && r < RY) {
                    const double* W = P.W[k];
                    if constexpr (S::ISO[k] != 0) {
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
        }(),
        ...);
}

template <class S, int BYT, int RY, int DX, int... Y>
__device__ __forceinline__ void column_rows(const StencilParams& P, const double* sm, int base, double* bx, double* by,
                                            double* bz, std::integer_sequence<int, Y...>) {
    using G = TileGeom<S, BYT, RY>;
    constexpr int ylo = shape_col_ymin<S>(DX);
    (
        [&] {
            constexpr int yy = ylo + Y;
            const int s = base + (yy + G::R) * G::PX + DX + G::R;
            row_accumulate<S, RY, DX, yy>(P, sm[s], sm[G::NS + s], sm[2 * G::NS + s], bx, by, bz,
                                          std::make_integer_sequence<int, S::K>{});
        }(),
        ...);
}

template <class S, int BYT, int RY, int... C>
__device__ __forceinline__ void all_columns(const StencilParams& P, const double* sm, int base, double* bx, double* by,
                                            double* bz, std::integer_sequence<int, C...>) {
    (
        [&] {
            constexpr int dx = C - S::R;
            constexpr int ylo = shape_col_ymin<S>(dx), yhi = shape_col_ymax<S>(dx);
            if constexpr (ylo <= yhi) {
                column_rows<S, BYT, RY, dx>(P, sm, base, bx, by, bz,
                                            std::make_integer_sequence<int, RY + yhi - ylo>{});
            }
        }(),
        ...);
}

template <int PASS>
__device__ __forceinline__ double epilogue(const DynCoef& C, const TiledArgs& A, int64_t i, int64_t N, double3 m0,
                                           const FieldOut& f, double3 hd) {
    const double3 B = make_double3(f.B.x - 2.0 * hd.x, f.B.y - 2.0 * hd.y, f.B.z - 2.0 * hd.z);
    if constexpr (PASS == PASS_FIELD) {
        if (A.out) st3(A.out, i, N, B);
        if (A.aux) A.aux[i] = site_energy(f, m0, hd);
        return total_energy_part(f, m0, hd);
    } else if constexpr (PASS == PASS_EULER) {
        const double3 D = llg_rhs(B, m0, C.alpha, C.inv_den);
        const double c = C.h_over_hbar;
        double3 t = make_double3(m0.x + D.x * c, m0.y + D.y * c, m0.z + D.z * c);
        if (C.thermal) {
            const double3 DT = llg_rhs(thermal_field(C, A.step, i, N), m0, C.alpha, C.inv_den);
            t = make_double3(t.x + DT.x * c, t.y + DT.y * c, t.z + DT.z * c);
        }
        st3(A.out, i, N, project(t, m0));
        return total_energy_part(f, m0, hd);
    } else if constexpr (PASS == PASS_HEUN1) {
        const double3 D = llg_rhs(B, m0, C.alpha, C.inv_den);
        const double c = C.h_over_hbar;
        const double3 t = make_double3(m0.x + D.x * c, m0.y + D.y * c, m0.z + D.z * c);
        st3(A.out, i, N, project(t, m0));
        st3(A.aux, i, N, D);
        if (C.thermal) st3(A.aux2, i, N, llg_rhs(thermal_field(C, A.step, i, N), m0, C.alpha, C.inv_den));
        return total_energy_part(f, m0, hd);
    } else if constexpr (PASS == PASS_HEUN2) {
        const double3 D2 = llg_rhs(B, m0, C.alpha, C.inv_den);
        const double3 d1 = ld3(A.aux, i, N);
        const double3 Di = make_double3(0.5 * d1.x + 0.5 * D2.x, 0.5 * d1.y + 0.5 * D2.y, 0.5 * d1.z + 0.5 * D2.z);
        const double c = C.h_over_hbar;
        double3 t = make_double3(m0.x + Di.x * c, m0.y + Di.y * c, m0.z + Di.z * c);
        if (C.thermal) {
            const double3 DT = ld3(A.aux2, i, N);
            t = make_double3(t.x + DT.x * c, t.y + DT.y * c, t.z + DT.z * c);
        }
        st3(A.out, i, N, project(t, m0));
        return 0.0;
    } else if constexpr (PASS == PASS_SIB1) {
        double3 H = B;
        if (C.thermal) {
            const double3 b = thermal_field(C, A.step, i, N);
            if (A.aux) st3(A.aux, i, N, b);  // the corrector reuses this step's draw
            H = make_double3(H.x + b.x, H.y + b.y, H.z + b.z);
        }
        const double3 y = sib_solve(m0, m0, H, C.alpha, C.sib_hc);
        st3(A.out, i, N, make_double3(0.5 * (m0.x + y.x), 0.5 * (m0.y + y.y), 0.5 * (m0.z + y.z)));
        return total_energy_part(f, m0, hd);
    } else {  // PASS_SIB2: m0 is the midpoint, the corrector starts from m_n
        double3 H = B;
        if (C.thermal) {
            const double3 b = A.aux ? ld3(A.aux, i, N) : thermal_field(C, A.step, i, N);
            H = make_double3(H.x + b.x, H.y + b.y, H.z + b.z);
        }
        const double3 mn = make_double3(A.mn[i], A.mn[N + i], A.mn[2 * N + i]);
        st3(A.out, i, N, sib_solve(mn, m0, H, C.alpha, C.sib_hc));
        return 0.0;
    }
}

template <class S, int BYT, int RY, int PASS>
__global__ void __launch_bounds__(32 * BYT) k_tiled(const __grid_constant__ StencilParams P, const DynCoef C,
                                                     const TiledArgs A) {
    using G = TileGeom<S, BYT, RY>;
    extern __shared__ double sm[];
    const int Lx = P.L[0], Ly = P.L[1];
    const int64_t layer = static_cast<int64_t>(Lx) * Ly;
    const int64_t N = layer * P.L[2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = tx + 32 * ty;
    const int x0 = blockIdx.x * G::TX, y0 = blockIdx.y * G::TY, z = blockIdx.z;
    const int64_t zoff = layer * z;
    const double* mx = A.ms + zoff;
    const double* my = A.ms + N + zoff;
    const double* mz = A.ms + 2 * N + zoff;
    // stage tile + halo; out-of-range sites of open axes are zero (no coupling)
    for (int idx = tid; idx < G::NS; idx += 32 * BYT) {
        const int ly = idx / G::PX;
        const int lx = idx - ly * G::PX;
        int gx = x0 + lx - G::R, gy = y0 + ly - G::R;
        bool ok = true;
        if (gx < 0 || gx >= Lx) {
            if (P.periodic[0]) gx = ((gx % Lx) + Lx) % Lx;
            else ok = false;
        }
        if (gy < 0 || gy >= Ly) {
            if (P.periodic[1]) gy = ((gy % Ly) + Ly) % Ly;
            else ok = false;
        }
        double vx = 0.0, vy = 0.0, vz = 0.0;
        if (ok) {
            const int64_t j = gx + static_cast<int64_t>(Lx) * gy;
            vx = __ldg(mx + j);
            vy = __ldg(my + j);
            vz = __ldg(mz + j);
        }
        sm[idx] = vx;
        sm[G::NS + idx] = vy;
        sm[2 * G::NS + idx] = vz;
    }
    __syncthreads();
    double bx[RY], by[RY], bz[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) bx[r] = by[r] = bz[r] = 0.0;
    const int base = (ty * RY) * G::PX + tx;
    all_columns<S, BYT, RY>(P, sm, base, bx, by, bz, std::make_integer_sequence<int, 2 * S::R + 1>{});
    double e = 0.0;
    const int x = x0 + tx;
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int y = y0 + ty * RY + r;
        const int c = base + (r + G::R) * G::PX + G::R;
        const double3 m0 = make_double3(sm[c], sm[G::NS + c], sm[2 * G::NS + c]);
        if (x < Lx && y < Ly) {
            const int64_t i = zoff + x + static_cast<int64_t>(Lx) * y;
            double b0 = bx[r], b1 = by[r], b2 = bz[r];
            if (P.has_onsite) {
                const double* W = P.W0;
                b0 = fma(W[0], m0.x, fma(W[1], m0.y, fma(W[2], m0.z, b0)));
                b1 = fma(W[3], m0.x, fma(W[4], m0.y, fma(W[5], m0.z, b1)));
                b2 = fma(W[6], m0.x, fma(W[7], m0.y, fma(W[8], m0.z, b2)));
            }
            FieldOut f;
            f.Bzee = make_double3(0.0, 0.0, 0.0);
            if (P.zee_on) {
                double3 b;
                if (A.bmap) b = make_double3(__ldg(A.bmap + i), __ldg(A.bmap + N + i), __ldg(A.bmap + 2 * N + i));
                else b = make_double3(P.bext[0], P.bext[1], P.bext[2]);
                f.Bzee = make_double3(P.zc * b.x, P.zc * b.y, P.zc * b.z);
            }
            f.B = make_double3(b0 + f.Bzee.x, b1 + f.Bzee.y, b2 + f.Bzee.z);
            const double3 hd = A.Hd.h ? ld_dip(A.Hd, x, y, z) : make_double3(0.0, 0.0, 0.0);
            e += epilogue<PASS>(C, A, i, N, m0, f, hd);
        }
    }
    if (A.R.out) {
        double v[1] = {e};
        grid_reduce<1>(v, A.R.partials, A.R.counter, A.R.out, A.R.nblocks);
    }
}

template <class S, int BYT, int RY>
struct TiledLauncher {
    using G = TileGeom<S, BYT, RY>;
    static dim3 grid(const StencilParams& P) {
        return dim3((P.L[0] + G::TX - 1) / G::TX, (P.L[1] + G::TY - 1) / G::TY, P.L[2]);
    }
    template <int PASS>
    static mj_status launch(const StencilParams& P, const DynCoef& C, const TiledArgs& A, cudaStream_t s) {
        static bool attr = false;
        auto kern = k_tiled<S, BYT, RY, PASS>;
        if (!attr) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(G::smem_bytes));
            attr = true;
        }
        kern<<<grid(P), dim3(32, BYT), G::smem_bytes, s>>>(P, C, A);
        return cuda_status(cudaGetLastError(), "k_tiled");
    }
};

template <class S, int BYT, int RY>
mj_status tiled_pass(int pass, const StencilParams& P, const DynCoef& C, const TiledArgs& A, cudaStream_t s) {
    using L = TiledLauncher<S, BYT, RY>;
    switch (pass) {
        case PASS_FIELD: return L::template launch<PASS_FIELD>(P, C, A, s);
        case PASS_EULER: return L::template launch<PASS_EULER>(P, C, A, s);
        case PASS_HEUN1: return L::template launch<PASS_HEUN1>(P, C, A, s);
        case PASS_HEUN2: return L::template launch<PASS_HEUN2>(P, C, A, s);
        case PASS_SIB1: return L::template launch<PASS_SIB1>(P, C, A, s);
        default: return L::template launch<PASS_SIB2>(P, C, A, s);
    }
}

// tile variants (threads in y, sites per thread); variant 0 is the default
template <class S>
mj_status tiled_dispatch(int variant, int pass, const StencilParams& P, const DynCoef& C, const TiledArgs& A,
                         cudaStream_t s) {
    switch (variant) {
        case 1: return tiled_pass<S, 8, 4>(pass, P, C, A, s);
        case 2: return tiled_pass<S, 4, 4>(pass, P, C, A, s);
        case 3: return tiled_pass<S, 2, 8>(pass, P, C, A, s);
        default: return tiled_pass<S, 4, 8>(pass, P, C, A, s);
    }
}

int64_t tiled_blocks(int shape, int variant, const StencilParams& P) {
    const int ty = variant == 1 ? 32 : variant == 2 ? 16 : variant == 3 ? 16 : 32;
    (void)shape;
    return static_cast<int64_t>((P.L[0] + 31) / 32) * ((P.L[1] + ty - 1) / ty) * P.L[2];
}

}  // namespace

int64_t tiled_energy_blocks(const mj_plan* p) { return tiled_blocks(p->sp.shape, p->tile_variant, p->sp); }

// pass: 0 field, 1 euler, 2 heun1, 3 heun2, 4 sib1, 5 sib2
mj_status launch_tiled(mj_plan* p, int pass, const DynCoef& C, const double* ms, const double* mn, double* out,
                       double* aux, double* aux2, DipView Hd, double* E_out, uint32_t step, cudaStream_t s) {
    TiledArgs A;
    A.ms = ms;
    A.mn = mn;
    A.out = out;
    A.aux = aux;
    A.aux2 = aux2;
    A.bmap = p->d_bmap;
    A.Hd = Hd;
    A.R.partials = p->d_partials;
    A.R.counter = p->d_counter;
    A.R.out = E_out;
    A.R.nblocks = static_cast<int>(tiled_energy_blocks(p));
    A.step = step;
    const int v = p->tile_variant;
    switch (p->sp.shape) {
        case kShapeSquareNN: return tiled_dispatch<ShapeSquareNN>(v, pass, p->sp, C, A, s);
        case kShapeSquare2: return tiled_dispatch<ShapeSquare2>(v, pass, p->sp, C, A, s);
        case kShapeTriNN: return tiled_dispatch<ShapeTriNN>(v, pass, p->sp, C, A, s);
        case kShapeTri3: return tiled_dispatch<ShapeTri3>(v, pass, p->sp, C, A, s);
        default: return set_error(MJ_ERR_ARG, "no tiled kernel for this stencil shape");
    }
}

}  // namespace mj
