// Shared-memory tiled stencil passes for the lattices with compile-time offset
// tables (mj_shapes.hpp): square NN / NN+NNN, triangular NN / three shells.
//
// A block of 32 x BYT threads owns a 32 x (BYT*RY) tile of one z-layer; each
// thread owns RY sites stacked along y.  The tile plus its halo is staged in
// shared memory (SoA), then each thread walks the stencil column by column: a
// value of column dx is loaded once and accumulated into every one of the
// thread's RY sites that sees it.  Offsets and tensor slots are compile-time
// constants; the coupling values come from the launch parameters.
//
// k_tiled stages the tile + halo either with plain loads (periodic wrap resolved
// per element) or with one cp.async.bulk.tensor (TMA, 4D box: x, y, z,
// component) completing on an mbarrier, while the threads compute the inputs
// of their epilogue (the thermal draw); on open axes the TMA zero fill of
// out-of-range cells is the open boundary, and the halo cells of a tile that
// wrap around a periodic edge are then rewritten with plain loads.  The halo
// along x is rounded up to an even width so that every TMA box starts on a
// 16-byte boundary.  No cluster multicast anywhere.
//
// Sparsity (template SP): with SP_AXIAL every anisotropic offset tensor has
// W[0][1] = W[1][0] = 0 (exchange plus a DMI vector in the lattice plane), the
// on-site tensor is zero but for W0[2][2] (uniaxial anisotropy along z) and a
// uniform applied field points along z; the kernels then skip the products with
// those zeros (7 instead of 9 per anisotropic neighbour, 1 instead of 9 on
// site).  SP_FULL is the general form.  The host picks the form per launch.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <type_traits>
#include <utility>

#include "mj_device.cuh"
#include "mj_internal.hpp"
#include "mj_shapes.hpp"

namespace mj {
namespace {

// PASS_GNEB: the field of GNEB images (a launch over nimg images), projected
// on each spin's tangent plane and stored, with each tile's six path sums and
// energy as block partials
enum { PASS_FIELD = 0, PASS_EULER = 1, PASS_HEUN1 = 2, PASS_HEUN2 = 3, PASS_SIB1 = 4, PASS_SIB2 = 5, PASS_GNEB = 6 };
enum { SP_FULL = 0, SP_AXIAL = 1 };

// Energy reduction of a launch.  mode 0: grid_reduce into `out` (if set);
// mode 1: write one partial per block, no ticket (the next pass sums them);
// mode 2: block 0 sums the `nblocks` partials of the previous pass into `out`.
struct TReduce {
    double* partials;
    unsigned int* counter;
    double* out;
    int nblocks;
    int mode;
};

struct TiledArgs {
    const double* ms;   // spins the stencil runs on (m, or the midpoint in pass 2)
    const double* mn;   // m_n (own site) for the SIB corrector
    double* out;        // field B / next state / midpoint
    double* aux;        // Heun D1, SIB Philox draw, or per-site energy (field pass)
    double* aux2;       // Heun DT
    const double* bmap; // per-cell applied field (SoA) or null
    DipView Hd;
    TReduce R;
    uint32_t step;
    int* status;        // device status word (bounded-wait timeouts)
    int ty0;            // first tile row of a launch over a range of tile rows
    int nty_all;        // tile rows of the whole lattice (0: the launch covers all of them)
    int ty_count;       // tile rows of this launch (host side: its grid height)
    int tma;            // 1: tile + halo staged by TMA through the kernel's tensor map
    int pdl;            // 1: launched as a programmatic dependent of the previous kernel
    int nimg;           // > 1: blockIdx.z runs over (image, layer) of nimg lattices stored
                        // back to back (3N doubles apart in ms / out, N in aux)
    int smem_bytes;     // host side: dynamic shared memory of the launch when above the
                        // tile's (caps the resident blocks per SM; the excess is unused)
    int img_up, img_dn; // PASS_GNEB, set per block: the image has a next / a previous one
};

// Programmatic dependent launch: a kernel lets the next one in its stream launch
// once all of its own blocks are resident (launch_dependents at its start), and
// reads what the previous kernel wrote only after griddepcontrol.wait, which
// returns once that kernel has completed with its memory visible.  Both are
// no-ops for a launch without the programmatic attribute.
__device__ __forceinline__ void pdl_allow_next() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_prev() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <class S, int BYT, int RY>
struct TileGeom {
    static constexpr int R = S::R;               // halo along y
    static constexpr int RX = (S::R + 1) & ~1;   // halo along x, even (16-byte TMA boxes)
    static constexpr int TX = 32, TY = BYT * RY;
    static constexpr int PX = TX + 2 * RX;
    static constexpr int PY = TY + 2 * R;
    static constexpr int NS = PX * PY;
    static constexpr size_t buf_bytes = sizeof(double) * 3 * NS;        // one TMA box
    static constexpr size_t buf_stride = (buf_bytes + 127) / 128 * 128;  // 128-byte aligned buffers
    static constexpr size_t buf_stride_d = buf_stride / sizeof(double);
};

// ---------------------------------------------------------------------------
// stencil accumulation, fully unrolled over compile-time offsets
template <class S, int RY, int DX, int YY, int SP, int... Kk>
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
                    } else if constexpr (SP == SP_AXIAL) {  // W[1] = W[3] = 0
                        bx[r] = fma(W[0], vx, fma(W[2], vz, bx[r]));
                        by[r] = fma(W[4], vy, fma(W[5], vz, by[r]));
                        bz[r] = fma(W[6], vx, fma(W[7], vy, fma(W[8], vz, bz[r])));
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

template <class S, int BYT, int RY, int DX, int SP, int... Y>
__device__ __forceinline__ void column_rows(const StencilParams& P, const double* sm, int base, double* bx, double* by,
                                            double* bz, std::integer_sequence<int, Y...>) {
    using G = TileGeom<S, BYT, RY>;
    constexpr int ylo = shape_col_ymin<S>(DX);
    (
        [&] {
            constexpr int yy = ylo + Y;
            const int s = base + (yy + G::R) * G::PX + DX + G::RX;
            row_accumulate<S, RY, DX, yy, SP>(P, sm[s], sm[G::NS + s], sm[2 * G::NS + s], bx, by, bz,
                                              std::make_integer_sequence<int, S::K>{});
        }(),
        ...);
}

template <class S, int BYT, int RY, int SP = SP_FULL, int... C>
__device__ __forceinline__ void all_columns(const StencilParams& P, const double* sm, int base, double* bx, double* by,
                                            double* bz, std::integer_sequence<int, C...>) {
    (
        [&] {
            constexpr int dx = C - S::R;
            constexpr int ylo = shape_col_ymin<S>(dx), yhi = shape_col_ymax<S>(dx);
            if constexpr (ylo <= yhi) {
                column_rows<S, BYT, RY, dx, SP>(P, sm, base, bx, by, bz,
                                                std::make_integer_sequence<int, RY + yhi - ylo>{});
            }
        }(),
        ...);
}

// Global loads of the staging and prefetch: CG = false takes the read-only
// path (data no block of the launch writes); CG = true caches at L2 only, for
// data written earlier in the same launch by other blocks (the fused step).
template <bool CG>
__device__ __forceinline__ double ldg_or_cg(const double* p) {
    if constexpr (CG) return __ldcg(p);
    return __ldg(p);
}

// per-site epilogue inputs that live in global memory, loaded before the
// stencil so that their latency overlaps it
struct Pre {
    double3 a;  // SIB2: m_n;  HEUN2: D1
    double3 b;  // SIB2: stored Philox draw;  HEUN2: DT
};

// The thermal draw of the passes that make one (Euler, Heun predictor, SIB
// predictor) is part of the prefetch: it depends on neither the tile nor the
// stencil, so it can run while the tile's halo loads are in flight.
template <int PASS, bool CG = false>
__device__ __forceinline__ Pre prefetch(const DynCoef& C, const TiledArgs& A, int64_t i, int64_t N) {
    Pre p;
    p.a = make_double3(0.0, 0.0, 0.0);
    p.b = p.a;
    if constexpr (PASS == PASS_SIB2) {
        p.a = make_double3(A.mn[i], A.mn[N + i], A.mn[2 * N + i]);
        if (C.thermal)
            p.b = A.aux ? make_double3(ldg_or_cg<CG>(A.aux + i), ldg_or_cg<CG>(A.aux + N + i),
                                       ldg_or_cg<CG>(A.aux + 2 * N + i))
                        : thermal_field(C, A.step, i, N);
    } else if constexpr (PASS == PASS_HEUN2) {
        p.a = ld3(A.aux, i, N);
        if (C.thermal) p.b = ld3(A.aux2, i, N);
    } else if constexpr (PASS == PASS_SIB1 || PASS == PASS_EULER || PASS == PASS_HEUN1) {
        if (C.thermal) p.b = thermal_field(C, A.step, i, N);
    }
    return p;
}

// Contribution of one site to H%energy: -m.Bmm/2 - m.Bzee (+ m.Hd with the dipolar
// term, counted once; fft_ham_base.f90:258-267), B = Bmm + Bzee the real-space field.
// ZAX: the Zeeman part points along z (its x, y parts are not added: IEEE
// arithmetic keeps x + 0 and x * 0 as operations).
template <bool HD, bool ZAX = false>
__device__ __forceinline__ double energy_part(double3 B, double3 Bzee, double3 m, double3 hd) {
    const double mz = ZAX ? m.z * Bzee.z : dot(m, Bzee);
    const double e = -0.5 * (dot(m, B) + mz);
    if constexpr (HD) return e + dot(m, hd);
    return e;
}

// The pass's update of one site.  B = the real-space field (MM + Zeeman), Bzee
// its Zeeman part, hd the dipolar H (HD); returns the site's energy part where
// the pass computes one.
template <int PASS, bool HD, bool ZAX = false>
__device__ __forceinline__ double epilogue(const DynCoef& C, const TiledArgs& A, int64_t i, int64_t N, double3 m0,
                                           double3 Brs, double3 Bzee, double3 hd, const Pre& pre) {
    double3 B = Brs;
    if constexpr (HD) B = make_double3(Brs.x - 2.0 * hd.x, Brs.y - 2.0 * hd.y, Brs.z - 2.0 * hd.z);
    if constexpr (PASS == PASS_FIELD) {
        if (A.out) st3(A.out, i, N, B);
        // per-site energy (energy_distrib, left-assigned; hamiltonian_collection.f90:332-363):
        // the dipolar term doubled as in fft_ham_base.f90:247-256
        if (A.aux) {
            double es = -0.5 * (dot(m0, Brs) + (ZAX ? m0.z * Bzee.z : dot(m0, Bzee)));
            if constexpr (HD) es += 2.0 * dot(m0, hd);
            A.aux[i] = es;
        }
        return energy_part<HD, ZAX>(Brs, Bzee, m0, hd);
    } else if constexpr (PASS == PASS_EULER) {
        const double3 D = llg_rhs(B, m0, C.alpha, C.inv_den);
        const double c = C.h_over_hbar;
        double3 t = make_double3(m0.x + D.x * c, m0.y + D.y * c, m0.z + D.z * c);
        if (C.thermal) {
            const double3 DT = llg_rhs(pre.b, m0, C.alpha, C.inv_den);
            t = make_double3(t.x + DT.x * c, t.y + DT.y * c, t.z + DT.z * c);
        }
        const double3 mo = project(t, m0);
        flag_nonfinite(A.status, mo);
        st3(A.out, i, N, mo);
        return energy_part<HD, ZAX>(Brs, Bzee, m0, hd);
    } else if constexpr (PASS == PASS_HEUN1) {
        const double3 D = llg_rhs(B, m0, C.alpha, C.inv_den);
        const double c = C.h_over_hbar;
        const double3 t = make_double3(m0.x + D.x * c, m0.y + D.y * c, m0.z + D.z * c);
        st3(A.out, i, N, project(t, m0));
        st3(A.aux, i, N, D);
        if (C.thermal) st3(A.aux2, i, N, llg_rhs(pre.b, m0, C.alpha, C.inv_den));
        return energy_part<HD, ZAX>(Brs, Bzee, m0, hd);
    } else if constexpr (PASS == PASS_HEUN2) {
        const double3 D2 = llg_rhs(B, m0, C.alpha, C.inv_den);
        const double3 d1 = pre.a;
        const double3 Di = make_double3(0.5 * d1.x + 0.5 * D2.x, 0.5 * d1.y + 0.5 * D2.y, 0.5 * d1.z + 0.5 * D2.z);
        const double c = C.h_over_hbar;
        double3 t = make_double3(m0.x + Di.x * c, m0.y + Di.y * c, m0.z + Di.z * c);
        if (C.thermal) {
            const double3 DT = pre.b;
            t = make_double3(t.x + DT.x * c, t.y + DT.y * c, t.z + DT.z * c);
        }
        const double3 mo = project(t, m0);
        flag_nonfinite(A.status, mo);
        st3(A.out, i, N, mo);
        return 0.0;
    } else if constexpr (PASS == PASS_SIB1) {
        double3 H = B;
        if (C.thermal) {
            const double3 b = pre.b;
            if (A.aux) st3(A.aux, i, N, b);  // the corrector reuses this step's draw
            H = make_double3(H.x + b.x, H.y + b.y, H.z + b.z);
        }
        st3(A.out, i, N, sib_solve<true>(m0, m0, H, C.alpha, C.sib_hc));
        return energy_part<HD, ZAX>(Brs, Bzee, m0, hd);
    } else {  // PASS_SIB2: m0 is the midpoint, the corrector starts from m_n
        double3 H = B;
        if (C.thermal) H = make_double3(H.x + pre.b.x, H.y + pre.b.y, H.z + pre.b.z);
        const double3 mo = sib_solve(pre.a, m0, H, C.alpha, C.sib_hc);
        flag_nonfinite(A.status, mo);
        st3(A.out, i, N, mo);
        return 0.0;
    }
}

// plain staging of tile + halo; periodic wrap per element, zeros off open edges
template <class S, int BYT, int RY, bool CG = false>
__device__ __forceinline__ void load_tile(const StencilParams& P, const double* ms, int x0, int y0, int z, double* sm) {
    using G = TileGeom<S, BYT, RY>;
    const int Lx = P.L[0], Ly = P.L[1];
    const int64_t layer = static_cast<int64_t>(Lx) * Ly;
    const int64_t N = layer * P.L[2];
    const double* mx = ms + layer * z;
    const int tid = threadIdx.x + 32 * threadIdx.y;
    for (int idx = tid; idx < G::NS; idx += 32 * BYT) {
        const int ly = idx / G::PX;
        const int lx = idx - ly * G::PX;
        int gx = x0 + lx - G::RX, gy = y0 + ly - G::R;
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
            vx = ldg_or_cg<CG>(mx + j);
            vy = ldg_or_cg<CG>(mx + N + j);
            vz = ldg_or_cg<CG>(mx + 2 * N + j);
        }
        sm[idx] = vx;
        sm[G::NS + idx] = vy;
        sm[2 * G::NS + idx] = vz;
    }
}

// After a TMA box landed with zeros outside the lattice: rewrite the halo cells
// that lie across a periodic edge with the wrapped spins (cells across an open
// edge keep the zeros).
template <class S, int BYT, int RY, bool CG = false>
__device__ __forceinline__ void patch_periodic_halo(const StencilParams& P, const double* ms, int x0, int y0, int z,
                                                    double* sm) {
    using G = TileGeom<S, BYT, RY>;
    const int Lx = P.L[0], Ly = P.L[1];
    const int64_t layer = static_cast<int64_t>(Lx) * Ly;
    const int64_t N = layer * P.L[2];
    const double* mx = ms + layer * z;
    const int tid = threadIdx.x + 32 * threadIdx.y;
    for (int idx = tid; idx < G::NS; idx += 32 * BYT) {
        const int ly = idx / G::PX;
        const int lx = idx - ly * G::PX;
        int gx = x0 + lx - G::RX, gy = y0 + ly - G::R;
        const bool outx = gx < 0 || gx >= Lx, outy = gy < 0 || gy >= Ly;
        if (!(outx || outy)) continue;                      // inside: the TMA copy holds it
        if ((outx && !P.periodic[0]) || (outy && !P.periodic[1])) continue;  // open edge: zero
        if (outx) gx = ((gx % Lx) + Lx) % Lx;
        if (outy) gy = ((gy % Ly) + Ly) % Ly;
        const int64_t j = gx + static_cast<int64_t>(Lx) * gy;
        sm[idx] = ldg_or_cg<CG>(mx + j);
        sm[G::NS + idx] = ldg_or_cg<CG>(mx + N + j);
        sm[2 * G::NS + idx] = ldg_or_cg<CG>(mx + 2 * N + j);
    }
}

// The same staging in two halves: the loads into registers, then the stores
// to shared memory, so that independent work can run while the loads are in
// flight.  Used when each thread stages at most kMaxStagedPerThread elements.
constexpr int kMaxStagedPerThread = 3;
template <class S, int BYT, int RY>
struct Staged {
    static constexpr int NT = 32 * BYT;
    static constexpr int NPT = (TileGeom<S, BYT, RY>::NS + NT - 1) / NT;
    double v[NPT][3];
};

template <class S, int BYT, int RY>
__device__ __forceinline__ void load_tile_issue(const StencilParams& P, const double* ms, int x0, int y0, int z,
                                                Staged<S, BYT, RY>& st) {
    using G = TileGeom<S, BYT, RY>;
    using T = Staged<S, BYT, RY>;
    const int Lx = P.L[0], Ly = P.L[1];
    const int64_t layer = static_cast<int64_t>(Lx) * Ly;
    const int64_t N = layer * P.L[2];
    const double* mx = ms + layer * z;
    const int tid = threadIdx.x + 32 * threadIdx.y;
#pragma unroll
    for (int k = 0; k < T::NPT; ++k) {
        const int idx = tid + k * T::NT;
        double vx = 0.0, vy = 0.0, vz = 0.0;
        if (idx < G::NS) {
            const int ly = idx / G::PX;
            const int lx = idx - ly * G::PX;
            int gx = x0 + lx - G::RX, gy = y0 + ly - G::R;
            bool ok = true;
            if (gx < 0 || gx >= Lx) {
                if (P.periodic[0]) gx = ((gx % Lx) + Lx) % Lx;
                else ok = false;
            }
            if (gy < 0 || gy >= Ly) {
                if (P.periodic[1]) gy = ((gy % Ly) + Ly) % Ly;
                else ok = false;
            }
            if (ok) {
                const int64_t j = gx + static_cast<int64_t>(Lx) * gy;
                vx = __ldg(mx + j);
                vy = __ldg(mx + N + j);
                vz = __ldg(mx + 2 * N + j);
            }
        }
        st.v[k][0] = vx;
        st.v[k][1] = vy;
        st.v[k][2] = vz;
    }
}

template <class S, int BYT, int RY>
__device__ __forceinline__ void load_tile_commit(const Staged<S, BYT, RY>& st, double* sm) {
    using G = TileGeom<S, BYT, RY>;
    using T = Staged<S, BYT, RY>;
    const int tid = threadIdx.x + 32 * threadIdx.y;
#pragma unroll
    for (int k = 0; k < T::NPT; ++k) {
        const int idx = tid + k * T::NT;
        if (idx < G::NS) {
            sm[idx] = st.v[k][0];
            sm[G::NS + idx] = st.v[k][1];
            sm[2 * G::NS + idx] = st.v[k][2];
        }
    }
}

// epilogue inputs of the thread's RY sites (see prefetch)
template <class S, int BYT, int RY, int PASS, bool CG = false>
__device__ __forceinline__ void prefetch_sites(const StencilParams& P, const DynCoef& C, const TiledArgs& A, int x0,
                                               int y0, int z, Pre* pre) {
    const int Lx = P.L[0], Ly = P.L[1];
    const int64_t layer = static_cast<int64_t>(Lx) * Ly;
    const int64_t N = layer * P.L[2];
    const int x = x0 + threadIdx.x;
    if constexpr (RY % 2 == 0 && (PASS == PASS_SIB1 || PASS == PASS_EULER || PASS == PASS_HEUN1)) {
        if (C.thermal && C.noise == MJ_NOISE_PHILOX) {
            // the draws of the thread's sites two at a time (a site past the
            // lattice's edge draws too and is not used)
#pragma unroll
            for (int r = 0; r < RY; r += 2) {
                const int y = y0 + threadIdx.y * RY + r;
                const int64_t i = layer * z + x + static_cast<int64_t>(Lx) * y;
                pre[r].a = pre[r + 1].a = make_double3(0.0, 0.0, 0.0);
                thermal_field_x2(C, A.step, i, i + Lx, pre[r].b, pre[r + 1].b);
            }
            return;
        }
    }
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int y = y0 + threadIdx.y * RY + r;
        if (x < Lx && y < Ly) pre[r] = prefetch<PASS, CG>(C, A, layer * z + x + static_cast<int64_t>(Lx) * y, N);
    }
}

// The epilogues of the thread's RY sites from the accumulated pair fields;
// ZMAP: per-cell applied field, HD: dipolar term.
template <class S, int BYT, int RY, int PASS, int SP, bool ZMAP, bool HD>
__device__ __forceinline__ double sites_epilogue(const StencilParams& P, const DynCoef& C, const TiledArgs& A,
                                                 const double* sm, int x0, int y0, int z, const Pre* pre,
                                                 const double* bx, const double* by, const double* bz,
                                                 double (&g6)[6]) {
    using G = TileGeom<S, BYT, RY>;
    const int Lx = P.L[0], Ly = P.L[1];
    const int64_t layer = static_cast<int64_t>(Lx) * Ly;
    const int64_t N = layer * P.L[2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = x0 + tx;
    const int base = (ty * RY) * G::PX + tx;
    double e = 0.0;
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int y = y0 + ty * RY + r;
        const int c = base + (r + G::R) * G::PX + G::RX;
        const double3 m0 = make_double3(sm[c], sm[G::NS + c], sm[2 * G::NS + c]);
        if (x < Lx && y < Ly) {
            const int64_t i = layer * z + x + static_cast<int64_t>(Lx) * y;
            double b0 = bx[r], b1 = by[r], b2 = bz[r];
            if (P.has_onsite) {
                const double* W = P.W0;
                if constexpr (SP == SP_AXIAL) {
                    b2 = fma(W[8], m0.z, b2);
                } else {
                    b0 = fma(W[0], m0.x, fma(W[1], m0.y, fma(W[2], m0.z, b0)));
                    b1 = fma(W[3], m0.x, fma(W[4], m0.y, fma(W[5], m0.z, b1)));
                    b2 = fma(W[6], m0.x, fma(W[7], m0.y, fma(W[8], m0.z, b2)));
                }
            }
            double3 Bzee = make_double3(0.0, 0.0, 0.0);
            if (P.zee_on) {
                if constexpr (ZMAP) {
                    Bzee = make_double3(P.zc * __ldg(A.bmap + i), P.zc * __ldg(A.bmap + N + i),
                                        P.zc * __ldg(A.bmap + 2 * N + i));
                } else if constexpr (SP == SP_AXIAL) {
                    Bzee.z = P.zc * P.bext[2];
                } else {
                    Bzee = make_double3(P.zc * P.bext[0], P.zc * P.bext[1], P.zc * P.bext[2]);
                }
            }
            constexpr bool ZAX = SP == SP_AXIAL && !ZMAP;
            const double3 Brs =
                ZAX ? make_double3(b0, b1, b2 + Bzee.z) : make_double3(b0 + Bzee.x, b1 + Bzee.y, b2 + Bzee.z);
            if constexpr (PASS == PASS_GNEB) {
                // the image's site energy (energy_distrib, as the field pass stores
                // it), the field projected on the tangent plane, the path sums
                e += -0.5 * (dot(m0, Brs) + (ZAX ? m0.z * Bzee.z : dot(m0, Bzee)));
                const double d = dot(Brs, m0);
                const double3 f = make_double3(Brs.x - d * m0.x, Brs.y - d * m0.y, Brs.z - d * m0.z);
                st3(A.out, i, N, f);
                const double3 mp = A.img_up ? ld3(A.ms + 3 * N, i, N) : m0;
                const double3 mm = A.img_dn ? ld3(A.ms - 3 * N, i, N) : m0;
                gneb_path_terms(m0, mp, mm, A.img_up != 0, f, g6);
            } else {
                double3 hd = make_double3(0.0, 0.0, 0.0);
                if constexpr (HD) hd = ld_dip(A.Hd, x, y, z);
                e += epilogue<PASS, HD, ZAX>(C, A, i, N, m0, Brs, Bzee, hd, pre[r]);
            }
        }
    }
    return e;
}

// stencil + epilogue of one staged tile; returns the energy of its sites
template <class S, int BYT, int RY, int PASS, int SP>
__device__ __forceinline__ double compute_tile(const StencilParams& P, const DynCoef& C, const TiledArgs& A,
                                               const double* sm, int x0, int y0, int z, const Pre* pre,
                                               double (&g6)[6]) {
    using G = TileGeom<S, BYT, RY>;
    double bx[RY], by[RY], bz[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) bx[r] = by[r] = bz[r] = 0.0;
    const int base = (threadIdx.y * RY) * G::PX + threadIdx.x;
    all_columns<S, BYT, RY, SP>(P, sm, base, bx, by, bz, std::make_integer_sequence<int, 2 * S::R + 1>{});
    // the branches are uniform over the launch; the GNEB images have no dipolar term
    if (A.bmap) {
        if constexpr (PASS != PASS_GNEB)
            if (A.Hd.h)
                return sites_epilogue<S, BYT, RY, PASS, SP, true, true>(P, C, A, sm, x0, y0, z, pre, bx, by, bz, g6);
        return sites_epilogue<S, BYT, RY, PASS, SP, true, false>(P, C, A, sm, x0, y0, z, pre, bx, by, bz, g6);
    }
    if constexpr (PASS != PASS_GNEB)
        if (A.Hd.h)
            return sites_epilogue<S, BYT, RY, PASS, SP, false, true>(P, C, A, sm, x0, y0, z, pre, bx, by, bz, g6);
    return sites_epilogue<S, BYT, RY, PASS, SP, false, false>(P, C, A, sm, x0, y0, z, pre, bx, by, bz, g6);
}

// ---------------------------------------------------------------------------
// TMA + mbarrier helpers (single CTA, no cluster multicast)
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false after ~limit polls (the caller records a timeout)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void tma_load_5d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y, int z,
                                            int c, int img) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
        "[%7];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(img), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y, int z,
                                            int c) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_u32(bar))
        : "memory");
}

// Poll limit of the wait for a tile's TMA copy (about 0.3 s with the 64 ns
// sleeps); far above any copy's latency.
constexpr uint32_t kTmaWaitPolls = 1u << 22;

template <class S, int BYT, int RY, int PASS, int MINB, int SP>
__global__ void __launch_bounds__(32 * BYT, MINB) k_tiled(const __grid_constant__ CUtensorMap tmap,
                                                     const __grid_constant__ StencilParams P, const DynCoef C,
                                                     const TiledArgs A0) {
    using G = TileGeom<S, BYT, RY>;
    extern __shared__ __align__(128) double smem_t[];
    __shared__ __align__(8) uint64_t bar;
    // a launch may cover the tile rows [ty0, ty0 + gridDim.y) of nty_all; block ids
    // (energy partials) are those of the launch over the whole lattice
    const int by = static_cast<int>(blockIdx.y) + A0.ty0;
    const int nty = A0.nty_all ? A0.nty_all : static_cast<int>(gridDim.y);
    int z = blockIdx.z, img = 0;
    TiledArgs A = A0;
    if (A0.nimg > 1) {  // image img of a launch over several lattices
        img = z / P.L[2];
        z -= img * P.L[2];
        const int64_t n = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
        A.ms += 3 * n * img;
        if (A.out) A.out += 3 * n * img;
        if (A.aux) A.aux += n * img;
    }
    A.img_up = img + 1 < A0.nimg ? 1 : 0;
    A.img_dn = img > 0 ? 1 : 0;
    const int x0 = blockIdx.x * G::TX, y0 = by * G::TY;
    const int bid = blockIdx.x + gridDim.x * (by + nty * blockIdx.z);
    const int tid = threadIdx.x + 32 * threadIdx.y;
    // the epilogue inputs of the passes that draw the thermal field depend on no
    // earlier kernel (an injected buffer is the caller's): computed before the
    // wait for the previous kernel, the others after it
    constexpr bool kPurePre = PASS == PASS_SIB1 || PASS == PASS_EULER || PASS == PASS_HEUN1 || PASS == PASS_FIELD;
    if (A.pdl) {
        pdl_allow_next();
        if constexpr (!kPurePre) pdl_wait_prev();
    }
    if (A.R.mode == 2 && bid == 0) ordered_sum<1>(A.R.partials, A.R.nblocks, A.R.out);
    Pre pre[RY];
    bool ok = true;
    if (A.tma) {
        // one copy of the whole box; the epilogue inputs (the thermal draw) are
        // computed while it is in flight
        if (tid == 0) {
            mbar_init(&bar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            if (A.pdl) pdl_wait_prev();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bar, static_cast<uint32_t>(G::buf_bytes));
            if (A.nimg > 1) tma_load_5d(&tmap, &bar, smem_t, x0 - G::RX, y0 - G::R, z, 0, img);
            else tma_load_4d(&tmap, &bar, smem_t, x0 - G::RX, y0 - G::R, z, 0);
        }
        prefetch_sites<S, BYT, RY, PASS>(P, C, A, x0, y0, z, pre);
        if (A.pdl) pdl_wait_prev();
        __syncthreads();  // the barrier's initialisation is visible to every waiting thread
        ok = mbar_wait_bounded(&bar, 0u, kTmaWaitPolls);
        if (__syncthreads_or(!ok)) {
            ok = false;
            if (tid == 0 && A.status) atomicOr(A.status, kStatusTimeout);
            // let the copy land before the block leaves (bounded), then only the
            // energy reduction below runs, so every block still takes part in it
            mbar_wait_bounded(&bar, 0u, 1u << 16);
        } else {
            const bool wraps = (P.periodic[0] && (x0 - G::RX < 0 || x0 + G::TX + G::RX > P.L[0])) ||
                               (P.periodic[1] && (y0 - G::R < 0 || y0 + G::TY + G::R > P.L[1]));
            if (wraps) {
                patch_periodic_halo<S, BYT, RY>(P, A.ms, x0, y0, z, smem_t);
                __syncthreads();
            }
        }
    } else if constexpr (Staged<S, BYT, RY>::NPT <= kMaxStagedPerThread) {
        // halo loads in flight while the epilogue inputs (the thermal draw) are computed
        Staged<S, BYT, RY> st;
        if (A.pdl) pdl_wait_prev();
        load_tile_issue<S, BYT, RY>(P, A.ms, x0, y0, z, st);
        prefetch_sites<S, BYT, RY, PASS>(P, C, A, x0, y0, z, pre);
        load_tile_commit<S, BYT, RY>(st, smem_t);
        __syncthreads();
    } else {
        if (A.pdl) pdl_wait_prev();
        load_tile<S, BYT, RY>(P, A.ms, x0, y0, z, smem_t);
        prefetch_sites<S, BYT, RY, PASS>(P, C, A, x0, y0, z, pre);
        __syncthreads();
    }
    double g6[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double e = ok ? compute_tile<S, BYT, RY, PASS, SP>(P, C, A, smem_t, x0, y0, z, pre, g6) : 0.0;
    if constexpr (PASS == PASS_GNEB) {  // the tile's path sums and energy, image-major
        double v[7] = {g6[0], g6[1], g6[2], g6[3], g6[4], g6[5], e};
        block_partials<7>(v, A.R.partials, A.R.nblocks, bid);
        return;
    }
    if (A.R.mode == 1) {
        double v[1] = {e};
        block_partials<1>(v, A.R.partials, A.R.nblocks, bid);
    } else if (A.R.mode == 0 && A.R.out) {
        double v[1] = {e};
        grid_reduce<1>(v, A.R.partials, A.R.counter, A.R.out, A.R.nblocks);
    }
}

// ---------------------------------------------------------------------------
// One SIB step in one launch (k_sib_fused).  The work items are tile rows of
// the predictor (P1) and of the corrector (P2) in a wavefront order per layer
// with a lag of L rows (L about the tile rows in flight at once, so that a
// corrector rarely finds its rows unfinished): P1 rows 0 .. L, then P1 row r
// followed by P2 row r-L for r = L+1 .. nty-1, then P2 rows nty-L .. nty-1 and
// 0 (each entry ntx tiles; one row: P1 then P2).  A corrector row r needs the
// predictor rows r-1, r, r+1 (across a periodic edge the row on the other
// side): all of them come earlier in the order.  Blocks take items from an
// atomic counter; a predictor tile counts itself into its row once its
// midpoint and draw are stored, and a corrector tile starts once its rows are
// complete.  Every row a corrector waits for was handed out before it, to a
// block that is running, so the waits end (they are bounded all the same), and
// the midpoint and draw are read back soon after they were written, from L2.
// No corrector tile's write of m overlaps a predictor tile still reading it (a
// corrector writes row r only after the predictor rows r-1 .. r+1 are done).
// The results equal the two-pass launches' bit for bit: the same tile code, the
// energy partials per predictor tile summed in tile order by the last block to
// finish, which also re-arms the scheduler words for the next launch.
struct FusedArgs {
    double* m;              // m_n in, m_{n+1} out
    double* mid;            // midpoint buffer
    double* draw;           // stored Philox draw (T > 0) or null
    const double* bmap;
    double* partials;       // energy partial per predictor tile
    double* E_out;          // energy of m_n or null
    unsigned int* sched;    // [0] work counter, [1] exit ticket, [2 ..) completed tiles per predictor row
    int* status;
    uint32_t step;
    int tma;                // stage by TMA through map_m / map_mid
    int lag;                // rows the corrector trails the predictor by (>= 1)
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

constexpr uint32_t kRowWaitPolls = 1u << 22;

// entry e (0 .. 2 nty - 1) of a layer's wavefront order: (corrector?, tile row)
__device__ __forceinline__ void wavefront_entry(int e, int nty, int lag_req, bool& corr, int& row) {
    if (nty == 1) {
        corr = e == 1;
        row = 0;
        return;
    }
    const int lag = lag_req < 1 ? 1 : (lag_req > nty - 1 ? nty - 1 : lag_req);
    const int a = lag + 1, b = 2 * (nty - 1 - lag);
    if (e < a) {  // P1 rows 0 .. lag
        corr = false;
        row = e;
    } else if (e < a + b) {  // P1 row r, then P2 row r - lag
        const int k = e - a;
        const int r = lag + 1 + (k >> 1);
        corr = (k & 1) != 0;
        row = corr ? r - lag : r;
    } else {  // P2 rows nty - lag .. nty - 1, then 0
        const int j = e - a - b;
        corr = true;
        row = j < lag ? nty - lag + j : 0;
    }
}

// Stage one tile (+ halo) of `src` into shared memory by TMA (with the
// periodic patch) or plain loads, computing the epilogue inputs meanwhile.
// Returns false when the copy's bounded wait gave up.
template <class S, int BYT, int RY, int PASS, bool CG>
__device__ __forceinline__ bool fused_stage(const CUtensorMap* map, const StencilParams& P, const DynCoef& C,
                                            const TiledArgs& A, bool tma, double* sm, uint64_t* bar, uint32_t& phase,
                                            int x0, int y0, int z, Pre* pre) {
    using G = TileGeom<S, BYT, RY>;
    const int tid = threadIdx.x + 32 * threadIdx.y;
    if (tma) {
        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar, static_cast<uint32_t>(G::buf_bytes));
            tma_load_4d(map, bar, sm, x0 - G::RX, y0 - G::R, z, 0);
        }
        prefetch_sites<S, BYT, RY, PASS, CG>(P, C, A, x0, y0, z, pre);
        const bool ok = mbar_wait_bounded(bar, phase, kTmaWaitPolls);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            mbar_wait_bounded(bar, phase ^ 1u, 1u << 16);  // let the copy land before leaving
            return false;
        }
        const bool wraps = (P.periodic[0] && (x0 - G::RX < 0 || x0 + G::TX + G::RX > P.L[0])) ||
                           (P.periodic[1] && (y0 - G::R < 0 || y0 + G::TY + G::R > P.L[1]));
        if (wraps) {
            patch_periodic_halo<S, BYT, RY, CG>(P, A.ms, x0, y0, z, sm);
            __syncthreads();
        }
        return true;
    }
    load_tile<S, BYT, RY, CG>(P, A.ms, x0, y0, z, sm);
    prefetch_sites<S, BYT, RY, PASS, CG>(P, C, A, x0, y0, z, pre);
    __syncthreads();
    return true;
}

// predictor tile t = (tx, ty, z): midpoint, draw and energy partial stored, row counted
template <class S, int BYT, int RY, int SP>
__device__ __forceinline__ bool fused_predictor(const CUtensorMap* map, const StencilParams& P, const DynCoef& C,
                                             const FusedArgs& F, double* sm, uint64_t* bar, uint32_t& phase, int tx,
                                             int ty, int z, int t, int T, unsigned int* row_done) {
    using G = TileGeom<S, BYT, RY>;
    TiledArgs A = {};
    A.bmap = F.bmap;
    A.step = F.step;
    A.status = F.status;
    A.ms = F.m;
    A.out = F.mid;
    A.aux = F.draw;
    const int x0 = tx * G::TX, y0 = ty * G::TY;
    Pre pre[RY];
    if (!fused_stage<S, BYT, RY, PASS_SIB1, false>(map, P, C, A, F.tma, sm, bar, phase, x0, y0, z, pre)) return false;
    double g6[6];
    const double e = compute_tile<S, BYT, RY, PASS_SIB1, SP>(P, C, A, sm, x0, y0, z, pre, g6);
    double v[1] = {e};
    block_partials<1>(v, F.partials, T, t);  // after the tile's stores
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        atomicAdd(row_done, 1u);
    }
    return true;
}

// corrector tile (tx, ty, z): m_{n+1} of the tile's sites, in place
template <class S, int BYT, int RY, int SP>
__device__ __forceinline__ bool fused_corrector(const CUtensorMap* map, const StencilParams& P, const DynCoef& C,
                                             const FusedArgs& F, double* sm, uint64_t* bar, uint32_t& phase, int tx,
                                             int ty, int z) {
    using G = TileGeom<S, BYT, RY>;
    TiledArgs A = {};
    A.bmap = F.bmap;
    A.step = F.step;
    A.status = F.status;
    A.ms = F.mid;
    A.mn = F.m;
    A.out = F.m;
    A.aux = F.draw;
    const int x0 = tx * G::TX, y0 = ty * G::TY;
    Pre pre[RY];
    if (!fused_stage<S, BYT, RY, PASS_SIB2, true>(map, P, C, A, F.tma, sm, bar, phase, x0, y0, z, pre)) return false;
    double g6[6];
    compute_tile<S, BYT, RY, PASS_SIB2, SP>(P, C, A, sm, x0, y0, z, pre, g6);
    return true;
}

template <class S, int BYT, int RY, int MINB, int SP>
__global__ void __launch_bounds__(32 * BYT, MINB) k_sib_fused(const __grid_constant__ CUtensorMap map_m,
                                                         const __grid_constant__ CUtensorMap map_mid,
                                                         const __grid_constant__ StencilParams P,
                                                         const __grid_constant__ DynCoef C,
                                                         const __grid_constant__ FusedArgs F) {
    using G = TileGeom<S, BYT, RY>;
    extern __shared__ __align__(128) double smem_t[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int s_item;
    __shared__ int s_ok;
    __shared__ bool s_last;
    const int tid = threadIdx.x + 32 * threadIdx.y;
    const int ntx = (P.L[0] + G::TX - 1) / G::TX, nty = (P.L[1] + G::TY - 1) / G::TY;
    const int T = ntx * nty * P.L[2];
    unsigned int* work = F.sched;
    unsigned int* ticket = F.sched + 1;
    unsigned int* rows = F.sched + 2;
    if (F.tma && tid == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase = 0u;
    for (;;) {
        if (tid == 0) s_item = static_cast<int>(atomicAdd(work, 1u));
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= 2 * T) break;
        const int tx = item % ntx;
        const int ent = item / ntx;
        const int z = ent / (2 * nty);
        bool corr;
        int ty;
        wavefront_entry(ent - z * 2 * nty, nty, F.lag, corr, ty);
        bool ok;
        if (!corr) {
            ok = fused_predictor<S, BYT, RY, SP>(&map_m, P, C, F, smem_t, &bar, phase, tx, ty, z,
                                                 tx + ntx * (ty + nty * z), T, rows + z * nty + ty);
        } else {
            // wait for the predictor rows the corrector's stencil reaches
            if (tid == 0) {
                int okw = 1;
                for (int d = -1; d <= 1 && okw; ++d) {
                    int r = ty + d;
                    if (r < 0 || r >= nty) {
                        if (!P.periodic[1] || nty < 2) continue;
                        r = (r + nty) % nty;
                    }
                    const unsigned int* w = rows + z * nty + r;
                    uint32_t it = 0;
                    while (ld_acquire_u32(w) < static_cast<unsigned int>(ntx)) {
                        if (++it > kRowWaitPolls) {
                            okw = 0;
                            break;
                        }
                        if (it > 32) __nanosleep(128);
                    }
                }
                __threadfence();
                asm volatile("fence.proxy.async.global;" ::: "memory");
                s_ok = okw;
            }
            __syncthreads();
            ok = s_ok != 0;
            if (ok) ok = fused_corrector<S, BYT, RY, SP>(&map_mid, P, C, F, smem_t, &bar, phase, tx, ty, z);
        }
        if (!ok) {
            if (tid == 0 && F.status) atomicOr(F.status, kStatusTimeout);
            break;
        }
        __syncthreads();  // the staging buffer is reused by the next item
    }
    // the last block to leave sums the energy partials and re-arms the scheduler
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (F.E_out) ordered_sum<1>(F.partials, T, F.E_out);
    const int nrows = nty * P.L[2];
    for (int r = tid; r < nrows; r += 32 * BYT) rows[r] = 0u;
    if (tid == 0) {
        *work = 0u;
        *ticket = 0u;
    }
}

// ---------------------------------------------------------------------------
template <class S, int BYT, int RY, int MINB>
struct TiledLauncher {
    using G = TileGeom<S, BYT, RY>;
    using Shape = S;
    static constexpr int BYT_ = BYT, RY_ = RY, MINB_ = MINB;
    static dim3 grid(const StencilParams& P) {
        return dim3((P.L[0] + G::TX - 1) / G::TX, (P.L[1] + G::TY - 1) / G::TY, P.L[2]);
    }
    template <int PASS, int SP>
    static mj_status launch(const CUtensorMap& map, const StencilParams& P, const DynCoef& C, const TiledArgs& A,
                            cudaStream_t s) {
        auto kern = k_tiled<S, BYT, RY, PASS, MINB, SP>;
        dim3 g = grid(P);
        if (A.nty_all) g.y = static_cast<unsigned>(A.ty_count);  // a range of tile rows
        if (A.nimg > 1) g.z *= static_cast<unsigned>(A.nimg);    // (image, layer)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = g;
        cfg.blockDim = dim3(32, BYT);
        cfg.dynamicSmemBytes = std::max<size_t>(G::buf_bytes, static_cast<size_t>(A.smem_bytes));
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = A.pdl ? 1 : 0;
        return cuda_status(cudaLaunchKernelEx(&cfg, kern, map, P, C, A), "k_tiled");
    }
    // the fused kernel holds both passes' code: a register cap of its own
    static constexpr int FMINB = RY <= 2 ? 768 / (32 * BYT) : 1;
    template <int SP>
    static mj_status launch_fused(const CUtensorMap& map_m, const CUtensorMap& map_mid, const StencilParams& P,
                                  const DynCoef& C, const FusedArgs& F, int num_sms, cudaStream_t s) {
        auto kern = k_sib_fused<S, BYT, RY, FMINB, SP>;
        static int per_sm = 0;  // resident blocks per SM (once per instantiation)
        if (per_sm <= 0) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * BYT, G::buf_bytes) != cudaSuccess ||
                per_sm <= 0)
                per_sm = 1;
        }
        const dim3 g = grid(P);
        const int64_t items = 2 * static_cast<int64_t>(g.x) * g.y * g.z;
        const int nb = static_cast<int>(std::min<int64_t>(items, static_cast<int64_t>(per_sm) * num_sms));
        FusedArgs Fl = F;
        Fl.lag = static_cast<int>((nb + g.x - 1) / g.x) + 1;  // tile rows in flight, plus one
        kern<<<nb, dim3(32, BYT), G::buf_bytes, s>>>(map_m, map_mid, P, C, Fl);
        return cuda_status(cudaGetLastError(), "k_sib_fused");
    }
};

template <class S, int BYT, int RY, int MINB, int SP>
mj_status tiled_pass_sp(int pass, const CUtensorMap& map, const StencilParams& P, const DynCoef& C, const TiledArgs& A,
                        cudaStream_t s) {
    using L = TiledLauncher<S, BYT, RY, MINB>;
    switch (pass) {
        case PASS_FIELD: return L::template launch<PASS_FIELD, SP>(map, P, C, A, s);
        case PASS_GNEB: return L::template launch<PASS_GNEB, SP>(map, P, C, A, s);
        case PASS_EULER: return L::template launch<PASS_EULER, SP>(map, P, C, A, s);
        case PASS_HEUN1: return L::template launch<PASS_HEUN1, SP>(map, P, C, A, s);
        case PASS_HEUN2: return L::template launch<PASS_HEUN2, SP>(map, P, C, A, s);
        case PASS_SIB1: return L::template launch<PASS_SIB1, SP>(map, P, C, A, s);
        default: return L::template launch<PASS_SIB2, SP>(map, P, C, A, s);
    }
}

template <class S, int BYT, int RY, int MINB>
mj_status tiled_pass(int pass, bool axial, const CUtensorMap& map, const StencilParams& P, const DynCoef& C,
                     const TiledArgs& A, cudaStream_t s) {
    if (axial) return tiled_pass_sp<S, BYT, RY, MINB, SP_AXIAL>(pass, map, P, C, A, s);
    return tiled_pass_sp<S, BYT, RY, MINB, SP_FULL>(pass, map, P, C, A, s);
}

// tile variants: (threads in y, sites per thread, min resident blocks per SM);
// the tile heights are kTiledVariantTY (mj_internal.hpp)
template <class S, class F>
auto with_variant(int variant, F&& f) {
    switch (variant) {
        case 1: return f(TiledLauncher<S, 8, 4, 1>{});
        case 2: return f(TiledLauncher<S, 8, 2, 1>{});
        case 3: return f(TiledLauncher<S, 4, 4, 6>{});
        case 4: return f(TiledLauncher<S, 8, 2, 4>{});
        case 5: return f(TiledLauncher<S, 4, 2, 8>{});
        default: return f(TiledLauncher<S, 4, 4, 1>{});
    }
}

// The sparsity form of a launch (SP_AXIAL when every zero it assumes holds).
template <class S>
bool stencil_axial(const StencilParams& sp, bool has_bmap) {
    for (int k = 0; k < S::K; ++k)
        if (S::ISO[k] == 0 && (sp.W[k][1] != 0.0 || sp.W[k][3] != 0.0)) return false;
    if (sp.has_onsite)
        for (int q = 0; q < 8; ++q)
            if (sp.W0[q] != 0.0) return false;
    if (sp.zee_on && !has_bmap && (sp.bext[0] != 0.0 || sp.bext[1] != 0.0)) return false;
    return true;
}

// ---------------------------------------------------------------------------
// tensor maps (driver entry point fetched through the runtime, no -lcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 4D map over the SoA spins: (x, y, z, component), box = tile + halo of one layer, 3 components
bool make_map(CUtensorMap* map, const double* base, const StencilParams& P, int box_x, int box_y) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (P.L[0] & 1) != 0) return false;
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(P.L[0]), static_cast<cuuint64_t>(P.L[1]),
                                static_cast<cuuint64_t>(P.L[2]), 3};
    const cuuint64_t layer = static_cast<cuuint64_t>(P.L[0]) * P.L[1];
    const cuuint64_t strides[3] = {static_cast<cuuint64_t>(P.L[0]) * 8, layer * 8, layer * P.L[2] * 8};
    const cuuint32_t box[4] = {static_cast<cuuint32_t>(box_x), static_cast<cuuint32_t>(box_y), 1, 3};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 5D map over nimg lattices stored back to back: (x, y, z, component, image)
bool make_map_images(CUtensorMap* map, const double* base, const StencilParams& P, int nimg, int box_x, int box_y) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (P.L[0] & 1) != 0) return false;
    const cuuint64_t layer = static_cast<cuuint64_t>(P.L[0]) * P.L[1];
    const cuuint64_t n = layer * P.L[2];
    const cuuint64_t dims[5] = {static_cast<cuuint64_t>(P.L[0]), static_cast<cuuint64_t>(P.L[1]),
                                static_cast<cuuint64_t>(P.L[2]), 3, static_cast<cuuint64_t>(nimg)};
    const cuuint64_t strides[4] = {static_cast<cuuint64_t>(P.L[0]) * 8, layer * 8, n * 8, 3 * n * 8};
    const cuuint32_t box[5] = {static_cast<cuuint32_t>(box_x), static_cast<cuuint32_t>(box_y), 1, 3, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// All passes of one compile-time shape (one translation unit per shape keeps
// the build parallel).  pass: 0 field, 1 euler, 2 heun1, 3 heun2, 4 sib1, 5 sib2
template <class S>
mj_status launch_tiled_shape(mj_plan* p, int pass, const DynCoef& C, const double* ms, const double* mn, double* out,
                             double* aux, double* aux2, DipView Hd, double* E_out, uint32_t step, cudaStream_t s,
                             int emode, int ty0, int nty) {
    TiledArgs A;
    std::memset(&A, 0, sizeof(A));
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
    A.R.mode = emode;
    if (emode == 2) A.R.nblocks = p->defer_nblocks;  // the partials of the previous pass
    A.step = step;
    A.status = p->d_status;
    const bool axial = stencil_axial<S>(p->sp, p->d_bmap != nullptr);
    return with_variant<S>(p->tile_variant, [&](auto L) -> mj_status {
        using Launcher = decltype(L);
        using G = typename Launcher::G;
        CUtensorMap map;
        std::memset(&map, 0, sizeof(map));
        if (nty >= 0) {  // tile rows [ty0, ty0 + nty) only, plain staging
            A.ty0 = ty0;
            A.nty_all = static_cast<int>(Launcher::grid(p->sp).y);
            A.ty_count = nty;
            if (nty == 0) return MJ_OK;
        } else {
            if (p->use_tma && make_map(&map, ms, p->sp, G::PX, G::PY)) A.tma = 1;
            A.pdl = p->use_pdl ? 1 : 0;
        }
        if (emode == 1) p->defer_nblocks = static_cast<int>(tiled_energy_blocks(p));
        A.smem_bytes = p->smem_cap_bytes;
        return tiled_pass<typename Launcher::Shape, Launcher::BYT_, Launcher::RY_, Launcher::MINB_>(pass, axial, map,
                                                                                                   p->sp, C, A, s);
    });
}

// One fused SIB step (predictor and corrector in one launch) of a 2D or layered
// lattice without the dipolar term; E_out receives the energy of m_n (or null).
template <class S>
mj_status launch_sib_fused_shape(mj_plan* p, const DynCoef& C, double* m, double* draw, double* E_out, uint32_t step,
                                 cudaStream_t s) {
    FusedArgs F;
    std::memset(&F, 0, sizeof(F));
    F.m = m;
    F.mid = p->d_mid;
    F.draw = draw;
    F.bmap = p->d_bmap;
    F.partials = p->d_partials;
    F.E_out = E_out;
    F.sched = p->d_sched;
    F.status = p->d_status;
    F.step = step;
    const bool axial = stencil_axial<S>(p->sp, p->d_bmap != nullptr);
    return with_variant<S>(p->tile_variant, [&](auto L) -> mj_status {
        using Launcher = decltype(L);
        using G = typename Launcher::G;
        CUtensorMap map_m, map_mid;
        std::memset(&map_m, 0, sizeof(map_m));
        std::memset(&map_mid, 0, sizeof(map_mid));
        if (p->use_tma && make_map(&map_m, m, p->sp, G::PX, G::PY) && make_map(&map_mid, p->d_mid, p->sp, G::PX, G::PY))
            F.tma = 1;
        p->defer_nblocks = static_cast<int>(tiled_energy_blocks(p));
        if (axial) return Launcher::template launch_fused<SP_AXIAL>(map_m, map_mid, p->sp, C, F, p->num_sms, s);
        return Launcher::template launch_fused<SP_FULL>(map_m, map_mid, p->sp, C, F, p->num_sms, s);
    });
}

// The GNEB images of a path held on the plan (nimg lattices back to back in m):
// per site the field projected on the spin's tangent plane into F, per tile the
// six path sums and the energy into partials[q nblocks + tile] (tiles image-major;
// *tiles_per_image receives the count).  No dipolar term.
template <class S>
mj_status launch_gneb_images_shape(mj_plan* p, const double* m, double* F, double* partials, int nimg,
                                   int64_t* tiles_per_image, cudaStream_t s) {
    TiledArgs A;
    std::memset(&A, 0, sizeof(A));
    A.ms = m;
    A.out = F;
    A.bmap = p->d_bmap;
    A.status = p->d_status;
    A.nimg = nimg;
    A.pdl = p->use_pdl ? 1 : 0;
    DynCoef C{};
    const bool axial = stencil_axial<S>(p->sp, p->d_bmap != nullptr);
    return with_variant<S>(p->tile_variant, [&](auto L) -> mj_status {
        using Launcher = decltype(L);
        using G = typename Launcher::G;
        const dim3 g = Launcher::grid(p->sp);
        *tiles_per_image = static_cast<int64_t>(g.x) * g.y * g.z;
        A.R.partials = partials;
        A.R.nblocks = static_cast<int>(*tiles_per_image * nimg);
        CUtensorMap map;
        std::memset(&map, 0, sizeof(map));
        if (p->use_tma && make_map_images(&map, m, p->sp, nimg, G::PX, G::PY)) A.tma = 1;
        return tiled_pass<typename Launcher::Shape, Launcher::BYT_, Launcher::RY_, Launcher::MINB_>(PASS_GNEB, axial,
                                                                                                   map, p->sp, C, A, s);
    });
}

}  // namespace
}  // namespace mj
