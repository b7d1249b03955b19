// Batched replicas: many independent lattices of one single-atom Hamiltonian
// (same cell, shells and couplings) with their own sizes, applied fields and
// temperatures, advanced together, one persistent launch per pass.
//
// Layout: the replicas' SoA spins are packed back to back, x[Ntot] | y[Ntot] |
// z[Ntot], replica r owning sites [off_r, off_r + Lx_r Ly_r).  A replica
// table (offset, size, Zeeman field, kT, Philox stream, temperature slot) and a
// tile list (replica, x0, y0), ordered by replica, drive persistent blocks that
// walk the tiles with a grid stride; each tile runs the same column-walking
// stencil as the single-lattice tiled kernels (mj_tiled_impl.cuh).  Per-replica
// energies are tile partials reduced in tile order (deterministic).
//
// Parallel tempering follows the reference's rule (paratemp-MC/paratemp.f90:
// 47-122): temperatures sit on a ladder of slots, neighbouring slots (l, l+1)
// are compared on alternating parities, delta = (1/kT_{l+1} - 1/kT_l)(E_{l+1} -
// E_l), accepted when delta > 0 or exp(max(delta, -200)) > u; an accepted swap
// exchanges the replicas' temperatures.  Here only neighbours of equal lattice
// size are compared, the uniform u is a Philox draw.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "mj_gneb.cuh"
#include "mj_mc.cuh"
#include "mj_tiled_impl.cuh"

namespace mj {

struct BatchRep {
    int64_t off;       // first packed site
    int Lx, Ly;
    int tile0, ntiles; // the replica's tiles in the tile list
    double zb[3];      // Zeeman field of the replica, zc * B_ext (eV)
    double kT;         // current temperature (eV), exchanged by the swaps
    uint32_t stream;   // Philox stream of the replica
    int slot;          // current temperature slot
};

namespace {

struct BatchArgs {
    const BatchRep* reps;
    const int4* tiles;  // (replica, x0, y0, -)
    int ntile;
    int64_t Ntot;
    const double* ms;   // stencil input (m or midpoint)
    const double* mn;   // m_n (SIB corrector)
    double* out;
    double* aux;        // stored Philox draw (SIB)
    double* tile_e;     // per-tile energy, null = none
    uint32_t step;
    double dt;          // SIB timestep (fs); sigma = sqrt(alpha kT hbar / dt) per replica
    int project;        // field pass: remove the component along m (B - (B.m) m)
    double* tile_g;     // GNEB pass: per-tile path sums (6 x ntile)
    int64_t gneb_n;     // GNEB pass: sites of an image (every replica one image)
    int gneb_nimg;      // GNEB pass: images
};

// BPASS_GNEB: the projected field pass with, per tile, the sums a GNEB iteration
// needs of every image r whatever the tangent's energy weights: with P the
// projection on the spin's tangent plane, A = P(m_{r+1} - m), B = P(m - m_{r-1})
// (zero at the path's ends), |A|^2, A.B, |B|^2, F.A, F.B and the squared angle
// to image r + 1; the energy-weighted tangent wp A + wm B then has |tau|^2 =
// wp^2 |A|^2 + 2 wp wm A.B + wm^2 |B|^2 and F.tau = wp F.A + wm F.B.
enum { BPASS_ENERGY = 0, BPASS_FIELD = 1, BPASS_GNEB = 2, BPASS_SIB1 = 4, BPASS_SIB2 = 5 };

template <class S, int BYT, int RY>
__device__ __forceinline__ void load_tile_b(const StencilParams& P, const BatchRep& R, const double* ms, int64_t Ntot,
                                            int x0, int y0, double* sm) {
    using G = TileGeom<S, BYT, RY>;
    const int Lx = R.Lx, Ly = R.Ly;
    const double* mx = ms + R.off;
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
            vx = __ldg(mx + j);
            vy = __ldg(mx + Ntot + j);
            vz = __ldg(mx + 2 * Ntot + j);
        }
        sm[idx] = vx;
        sm[G::NS + idx] = vy;
        sm[2 * G::NS + idx] = vz;
    }
}

// SP_AXIAL: the stencil's and the on-site term's zeros of the axial form (as
// the single-lattice tiled kernels; every replica's field then points along z).
template <class S, int BYT, int RY, int PASS, int SP = SP_FULL>
__device__ __forceinline__ double compute_tile_b(const StencilParams& P, const DynCoef& C, const BatchArgs& A,
                                                 const BatchRep& R, int rep, const double* sm, int x0, int y0,
                                                 double (&gs)[6]) {
    using G = TileGeom<S, BYT, RY>;
    const int64_t Nt = A.Ntot;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = x0 + tx;
    // same expression and thermal condition as the single-lattice coefficients
    const bool thermal = C.thermal && (R.kT * C.alpha > 1e-10) && (R.kT > 1e-8);
    const double sigma = thermal ? sqrt(C.alpha * R.kT * kHbar / A.dt) : 0.0;
    Pre pre[RY];
    if constexpr (PASS == BPASS_SIB2) {
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            const int y = y0 + ty * RY + r;
            if (x < R.Lx && y < R.Ly) {
                const int64_t i = R.off + x + static_cast<int64_t>(R.Lx) * y;
                pre[r].a = make_double3(A.mn[i], A.mn[Nt + i], A.mn[2 * Nt + i]);
                pre[r].b = thermal ? ld3(A.aux, i, Nt) : make_double3(0.0, 0.0, 0.0);
            }
        }
    } else if constexpr (PASS == BPASS_SIB1 && RY % 2 == 0) {
        // the thermal draws of the thread's sites, two at a time (a site past the
        // replica's edge draws too and is not used)
        if (thermal) {
#pragma unroll
            for (int r = 0; r < RY; r += 2) {
                const int64_t li = x + static_cast<int64_t>(R.Lx) * (y0 + ty * RY + r);
                double3 z0, z1;
                philox_normals_x2(C.keys, C.noise_tab, A.step, C.stream_id + R.stream, static_cast<uint32_t>(li),
                                  static_cast<uint32_t>(li + R.Lx), z0, z1);
                pre[r].b = make_double3(sigma * z0.x, sigma * z0.y, sigma * z0.z);
                pre[r + 1].b = make_double3(sigma * z1.x, sigma * z1.y, sigma * z1.z);
            }
        }
    }
    double bx[RY], by[RY], bz[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) bx[r] = by[r] = bz[r] = 0.0;
    const int base = (ty * RY) * G::PX + tx;
    all_columns<S, BYT, RY, SP>(P, sm, base, bx, by, bz, std::make_integer_sequence<int, 2 * S::R + 1>{});
    double e = 0.0;
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int y = y0 + ty * RY + r;
        const int c = base + (r + G::R) * G::PX + G::RX;
        const double3 m0 = make_double3(sm[c], sm[G::NS + c], sm[2 * G::NS + c]);
        if (x < R.Lx && y < R.Ly) {
            const int64_t li = x + static_cast<int64_t>(R.Lx) * y;  // site index within the replica
            const int64_t i = R.off + li;
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
            FieldOut f;
            f.Bzee = make_double3(R.zb[0], R.zb[1], R.zb[2]);
            f.B = make_double3(b0 + f.Bzee.x, b1 + f.Bzee.y, b2 + f.Bzee.z);
            const double3 zero = make_double3(0.0, 0.0, 0.0);
            if constexpr (PASS == BPASS_ENERGY) {
                e += total_energy_part(f, m0, zero);
            } else if constexpr (PASS == BPASS_FIELD || PASS == BPASS_GNEB) {
                e += total_energy_part(f, m0, zero);
                double3 Bv = f.B;
                if (PASS == BPASS_GNEB || A.project) {
                    const double d = dot(Bv, m0);
                    Bv = make_double3(Bv.x - d * m0.x, Bv.y - d * m0.y, Bv.z - d * m0.z);
                }
                st3(A.out, i, Nt, Bv);
                if constexpr (PASS == BPASS_GNEB) {
                    const bool up = rep + 1 < A.gneb_nimg, down = rep > 0;
                    const double3 mp = up ? ld3(A.ms, i + A.gneb_n, Nt) : m0;
                    const double3 mm = down ? ld3(A.ms, i - A.gneb_n, Nt) : m0;
                    double3 u = make_double3(mp.x - m0.x, mp.y - m0.y, mp.z - m0.z);
                    double3 w = make_double3(m0.x - mm.x, m0.y - mm.y, m0.z - mm.z);
                    const double du = dot(u, m0), dw = dot(w, m0);
                    u = make_double3(u.x - du * m0.x, u.y - du * m0.y, u.z - du * m0.z);
                    w = make_double3(w.x - dw * m0.x, w.y - dw * m0.y, w.z - dw * m0.z);
                    gs[0] += dot(u, u);
                    gs[1] += dot(u, w);
                    gs[2] += dot(w, w);
                    gs[3] += dot(Bv, u);
                    gs[4] += dot(Bv, w);
                    if (up) {
                        const double3 c = cross(m0, mp);
                        const double l = atan2(sqrt(dot(c, c)), dot(m0, mp));
                        gs[5] += l * l;
                    }
                }
            } else if constexpr (PASS == BPASS_SIB1) {
                e += total_energy_part(f, m0, zero);
                double3 H = f.B;
                if (thermal) {
                    double3 b;
                    if constexpr (RY % 2 == 0) {
                        b = pre[r].b;
                    } else {
                        const double3 z = philox_normals_tab(C.keys, C.noise_tab, A.step, C.stream_id + R.stream,
                                                             static_cast<uint32_t>(li));
                        b = make_double3(sigma * z.x, sigma * z.y, sigma * z.z);
                    }
                    st3(A.aux, i, Nt, b);
                    H = make_double3(H.x + b.x, H.y + b.y, H.z + b.z);
                }
                st3(A.out, i, Nt, sib_solve<true>(m0, m0, H, C.alpha, C.sib_hc));
            } else {
                double3 H = f.B;
                if (thermal) H = make_double3(H.x + pre[r].b.x, H.y + pre[r].b.y, H.z + pre[r].b.z);
                st3(A.out, i, Nt, sib_solve(pre[r].a, m0, H, C.alpha, C.sib_hc));
            }
        }
    }
    return e;
}

template <class S, int BYT, int RY, int MINB, int PASS, int SP>
__global__ void __launch_bounds__(32 * BYT, MINB) k_batch(const __grid_constant__ StencilParams P, const DynCoef C,
                                                           const BatchArgs A) {
    using G = TileGeom<S, BYT, RY>;
    extern __shared__ __align__(128) double smem_b[];
    // per tile: the energy, and for the GNEB pass its six path sums
    constexpr int NV = PASS == BPASS_GNEB ? 7 : 1;
    __shared__ double wsum[NV][8];
    BatchArgs Ar = A;
    if (C.step_base) Ar.step = A.step + *C.step_base;
    const int tid = threadIdx.x + 32 * threadIdx.y;
    for (int t = blockIdx.x; t < A.ntile; t += gridDim.x) {
        const int4 tl = A.tiles[t];
        const BatchRep R = A.reps[tl.x];
        load_tile_b<S, BYT, RY>(P, R, A.ms, A.Ntot, tl.y, tl.z, smem_b);
        __syncthreads();
        double v[NV];
        double gs[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        v[0] = compute_tile_b<S, BYT, RY, PASS, SP>(P, C, Ar, R, tl.x, smem_b, tl.y, tl.z, gs);
#pragma unroll
        for (int q = 1; q < NV; ++q) v[q] = gs[q - 1];
        if (A.tile_e) {
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                double e = v[q];
                for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
                if ((tid & 31) == 0) wsum[q][tid >> 5] = e;
            }
        }
        __syncthreads();  // tile buffer and wsum are reused by the next tile
        if (A.tile_e && tid == 0) {
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                double s = 0.0;
                for (int w = 0; w < BYT; ++w) s += wsum[q][w];
                if (q == 0) A.tile_e[t] = s;
                else A.tile_g[static_cast<int64_t>(q - 1) * A.ntile + t] = s;
            }
        }
    }
}

// per-replica energies: tile partials summed in tile order, one block per replica
__global__ void k_batch_energy(const BatchRep* reps, int nrep, const double* tile_e, double* E) {
    const int r = blockIdx.x;
    if (r >= nrep) return;
    __shared__ double part[256];
    const BatchRep R = reps[r];
    double s = 0.0;
    for (int t = threadIdx.x; t < R.ntiles; t += blockDim.x) s += tile_e[R.tile0 + t];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int k = 0; k < static_cast<int>(blockDim.x); ++k) tot += part[k];
        E[r] = tot;
    }
}

// one parallel-tempering round on the temperature ladder (single block)
// (C carries the Philox key schedule by value and, in a graph, the device step counter)
__global__ void k_pt_swap(BatchRep* reps, int* image, const double* slot_kT, int nslot, const double* E,
                          const DynCoef C, uint32_t round_base, uint32_t swap_every, int* nswap_accept) {
    uint32_t round = round_base;
    if (C.step_base) round += *C.step_base / swap_every;
    const int start = static_cast<int>(round & 1u);
    for (int l = start + 2 * static_cast<int>(threadIdx.x); l + 1 < nslot; l += 2 * static_cast<int>(blockDim.x)) {
        const int a = image[l], b = image[l + 1];
        const BatchRep Ra = reps[a], Rb = reps[b];
        if (Ra.Lx != Rb.Lx || Ra.Ly != Rb.Ly) continue;  // only neighbours of equal size
        const double delta = (1.0 / slot_kT[l + 1] - 1.0 / slot_kT[l]) * (E[b] - E[a]);
        bool acc = delta > 0.0;
        if (!acc) {
            uint32_t c[4] = {static_cast<uint32_t>(l), round, 0x50545357u /* "PTSW" */, 2u};
            philox10k(c, C.keys);
            acc = exp(fmax(delta, -200.0)) > u53(c[0], c[1]);
        }
        if (acc) {
            image[l] = b;
            image[l + 1] = a;
            reps[b].kT = slot_kT[l];
            reps[b].slot = l;
            reps[a].kT = slot_kT[l + 1];
            reps[a].slot = l + 1;
            if (nswap_accept) atomicAdd(nswap_accept + l, 1);
        }
    }
}

// ---------------------------------------------------------------------------
// Monte Carlo on the replicas (paratemp-MC/parallel_tempering.f90:163-181): each
// replica is a chain of its own (its own cone and counts, Philox stream
// stream_id + r, its site index within the replica), moved colour by colour at
// the temperature its ladder slot holds; the moves are mj_mc.cuh's.  MC tiles
// are (replica, tx block, ty block) of 32 x kMcBY threads over a colour class.
struct BatchMcArgs {
    const double* tab;          // sin/cos tables
    const BatchRep* reps;
    const int4* tiles;          // (replica, x block, y block, -)
    int64_t Ntot;
    double* m;
    const double* cos_cone;     // per replica
    unsigned long long* acc;    // accepted moves per replica
    uint32_t keys[20];
    int proposal;
    uint32_t sweep;
    uint32_t stream_id;
    McClass K;
};

template <class S>
__global__ void __launch_bounds__(32 * kMcBY, 8) k_batch_mc(const __grid_constant__ StencilParams P,
                                                  const __grid_constant__ BatchMcArgs A) {
    const int4 tl = A.tiles[blockIdx.x];
    const BatchRep R = A.reps[tl.x];
    const McClass& K = A.K;
    const int y = K.ry + K.sy * (tl.z * kMcBY + static_cast<int>(threadIdx.y));
    const int z = K.rz;  // replicas are one layer thick
    const int x = mc_class_x(K, y, z, tl.y * 32 + static_cast<int>(threadIdx.x));
    bool acc = false;
    if (x < R.Lx && y < R.Ly && z == 0) {
        double* mr = A.m + R.off;
        const int64_t li = x + static_cast<int64_t>(R.Lx) * y;
        const double3 s = ld3(mr, li, A.Ntot);
        const double3 Pf = pair_field<S>(P, mr, A.Ntot, R.Lx, R.Ly, 1, x, y, 0);
        double3 sn;
        double dE;
        acc = mc_move(P, A.keys, A.tab, A.proposal, R.kT, R.kT > 0.0 ? 1.0 / R.kT : 0.0, A.cos_cone[tl.x],
                      static_cast<uint32_t>(li), A.sweep, A.stream_id + R.stream, s, Pf,
                      make_double3(R.zb[0], R.zb[1], R.zb[2]), sn, dE);
        if (acc) st3(mr, li, A.Ntot, sn);
    }
    const int n = __syncthreads_count(acc);
    if (threadIdx.x == 0 && threadIdx.y == 0 && n) atomicAdd(A.acc + tl.x, static_cast<unsigned long long>(n));
}

// after a sweep: proposed counts, the cone rule of sample_sphere (track_value.f90
// cone_update, +-1e-4 per move of the sweep toward a running rate of 0.5, cone in
// [0.01, pi]) when adapting, and the cosine the next sweep uses
__global__ void k_batch_mc_cone(const BatchRep* reps, int nrep, const unsigned long long* acc, long long* prop,
                                double* cone, double* cos_cone, int adapt) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrep) return;
    const long long n = static_cast<long long>(reps[r].Lx) * reps[r].Ly;
    prop[r] += n;
    if (adapt) {
        const double rate = static_cast<double>(acc[r]) / static_cast<double>(prop[r]);
        // product and sum rounded apart (no fused multiply-add), as the host rule rounds them
        const double step = __dmul_rn(1e-4, static_cast<double>(n));
        double c = cone[r];
        if (rate > 0.5 && c < kPi) c = fmin(kPi, __dadd_rn(c, step));
        else if (rate < 0.5 && c > 0.01) c = fmax(0.01, __dsub_rn(c, step));
        cone[r] = c;
    }
    cos_cone[r] = cos(cone[r]);
}

__global__ void k_batch_mc_init(int nrep, double cone0, unsigned long long* acc, long long* prop, double* cone,
                                double* cos_cone) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrep) return;
    acc[r] = 0ull;
    prop[r] = 0ll;
    cone[r] = cone0;
    cos_cone[r] = cos(cone0);
}

// summed spins of each replica (one block per replica, fixed order) and its slot
__global__ void __launch_bounds__(256) k_batch_magnet(const BatchRep* reps, const double* m, int64_t Ntot, double* M,
                                                      int* slot) {
    const int r = blockIdx.x;
    const BatchRep R = reps[r];
    const int64_t n = static_cast<int64_t>(R.Lx) * R.Ly;
    double v[3] = {0.0, 0.0, 0.0};
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        v[0] += m[R.off + i];
        v[1] += m[Ntot + R.off + i];
        v[2] += m[2 * Ntot + R.off + i];
    }
    if (M) block_partials<3>(v, M + 3 * static_cast<int64_t>(r), 1, 0);
    if (slot && threadIdx.x == 0) slot[r] = R.slot;
}

// ---------------------------------------------------------------------------
// GNEB on the replicas taken as the images of one path (all of one size n, image
// r at sites [r n, (r + 1) n) of every component block): the kernels and the
// relaxation driver are in mj_gneb.cuh; the batch adds the fused GNEB field
// pass (BPASS_GNEB, the path sums per tile) and k_gneb_img.

// Per image r (one block each): the energy and the six path sums of the GNEB
// field pass, each summed over the image's tiles in tile order as
// k_batch_energy sums the energies (thread t the tiles t, t + 256, ...; then
// those partials in thread order, the all-zero ones beyond the image's tile
// count left out), into E[r] and img[q nrep + r]; the seven sums side by side.
__global__ void __launch_bounds__(256) k_gneb_img(const BatchRep* reps, int nrep, const double* __restrict__ tile_e,
                                                  const double* __restrict__ tile_g, int ntile, double* E,
                                                  double* img, const GnebCtl* ctl) {
    if (ctl->done) return;
    const int r = blockIdx.x;
    __shared__ double part[7][256];
    const BatchRep R = reps[r];
    for (int q = 0; q < 7; ++q) {
        const double* src = q == 0 ? tile_e : tile_g + static_cast<int64_t>(q - 1) * ntile;
        double s = 0.0;
        for (int t = threadIdx.x; t < R.ntiles; t += blockDim.x) s += src[R.tile0 + t];
        part[q][threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        const int q = threadIdx.x;
        const int nk = min(R.ntiles, static_cast<int>(blockDim.x));
        double tot = 0.0;
        for (int k = 0; k < nk; ++k) tot += part[q][k];
        if (q == 0) E[r] = tot;
        else img[(q - 1) * nrep + r] = tot;
    }
}

template <class S, int BYT, int RY, int MINB>
struct BatchLauncher {
    using G = TileGeom<S, BYT, RY>;
    static constexpr int TY = G::TY;
    template <int PASS, int SP>
    static mj_status launch(const StencilParams& P, const DynCoef& C, const BatchArgs& A, int nblocks, cudaStream_t s) {
        k_batch<S, BYT, RY, MINB, PASS, SP><<<nblocks, dim3(32, BYT), G::buf_bytes, s>>>(P, C, A);
        return cuda_status(cudaGetLastError(), "k_batch");
    }
    // the dynamics and energy passes in the axial form where it holds; the
    // field and GNEB passes in the full form
    static mj_status pass(int ps, bool axial, const StencilParams& P, const DynCoef& C, const BatchArgs& A,
                          int nblocks, cudaStream_t s) {
        switch (ps) {
            case BPASS_SIB1:
                return axial ? launch<BPASS_SIB1, SP_AXIAL>(P, C, A, nblocks, s)
                             : launch<BPASS_SIB1, SP_FULL>(P, C, A, nblocks, s);
            case BPASS_SIB2:
                return axial ? launch<BPASS_SIB2, SP_AXIAL>(P, C, A, nblocks, s)
                             : launch<BPASS_SIB2, SP_FULL>(P, C, A, nblocks, s);
            case BPASS_FIELD: return launch<BPASS_FIELD, SP_FULL>(P, C, A, nblocks, s);
            case BPASS_GNEB: return launch<BPASS_GNEB, SP_FULL>(P, C, A, nblocks, s);
            default:
                return axial ? launch<BPASS_ENERGY, SP_AXIAL>(P, C, A, nblocks, s)
                             : launch<BPASS_ENERGY, SP_FULL>(P, C, A, nblocks, s);
        }
    }
};

// batch tile variants: (threads in y, sites per thread, min resident blocks per SM)
constexpr int kBatchVariants = 5;
constexpr int kBatchTY[kBatchVariants] = {16, 16, 32, 8, 16};

template <class S>
mj_status batch_pass_shape(int variant, int ps, bool zaxial, const StencilParams& P, const DynCoef& C,
                           const BatchArgs& A, int nblocks, cudaStream_t s) {
    // axial: the stencil's zeros hold and every replica's field points along z
    const bool axial = zaxial && stencil_axial<S>(P, true);
    switch (variant) {
        case 1: return BatchLauncher<S, 8, 2, 1>::pass(ps, axial, P, C, A, nblocks, s);
        case 2: return BatchLauncher<S, 8, 4, 1>::pass(ps, axial, P, C, A, nblocks, s);
        case 3: return BatchLauncher<S, 4, 2, 8>::pass(ps, axial, P, C, A, nblocks, s);
        case 4: return BatchLauncher<S, 8, 2, 4>::pass(ps, axial, P, C, A, nblocks, s);
        default: return BatchLauncher<S, 4, 4, 1>::pass(ps, axial, P, C, A, nblocks, s);
    }
}

mj_status batch_pass(int shape, int variant, int ps, bool zaxial, const StencilParams& P, const DynCoef& C,
                     const BatchArgs& A, int nblocks, cudaStream_t s) {
    switch (shape) {
        case kShapeSquareNN: return batch_pass_shape<ShapeSquareNN>(variant, ps, zaxial, P, C, A, nblocks, s);
        case kShapeSquare2: return batch_pass_shape<ShapeSquare2>(variant, ps, zaxial, P, C, A, nblocks, s);
        case kShapeTriNN: return batch_pass_shape<ShapeTriNN>(variant, ps, zaxial, P, C, A, nblocks, s);
        case kShapeTri3: return batch_pass_shape<ShapeTri3>(variant, ps, zaxial, P, C, A, nblocks, s);
        default: return set_error(MJ_ERR_UNSUPPORTED, "batches need a tiled lattice shape");
    }
}

}  // namespace
}  // namespace mj

// ---------------------------------------------------------------------------
struct mj_batch {
    int device = 0;
    int nrep = 0;
    int64_t Ntot = 0;
    mj::StencilParams sp{};
    int shape = 0;
    int variant = 0;
    int blocks_per_sm = 8;
    bool zaxial = false;              // every replica's Zeeman field along z
    int num_sms = 148;
    std::vector<mj::BatchRep> reps;   // host copy (initial table)
    std::vector<int> L;               // 2*nrep
    std::vector<double> slot_kT;      // ladder of temperatures (eV), ascending
    int ntile = 0;
    double* d_m = nullptr;
    double* d_mid = nullptr;
    double* d_aux = nullptr;
    double* d_tile_e = nullptr;
    double* d_E = nullptr;
    double* d_slot_kT = nullptr;
    double* d_noise_tab = nullptr;
    mj::BatchRep* d_reps = nullptr;
    int4* d_tiles = nullptr;
    int* d_image = nullptr;
    int* d_accept = nullptr;
    uint32_t* d_stepctr = nullptr;
    double* d_stage = nullptr;
    double* d_gneb_part = nullptr;    // tangent norms: one partial per (image, block)
    // Monte Carlo: the colouring, its MC tile list, per-replica chain state
    int mc_col[4] = {0, 0, 0, 0};
    int4* d_mc_tiles = nullptr;
    int mc_ntile = 0;
    unsigned long long* d_mc_acc = nullptr;
    long long* d_mc_prop = nullptr;
    double* d_mc_cone = nullptr;
    double* d_mc_cos = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::string graph_key;
};

namespace mj {
namespace {

void batch_free(mj_batch* b) {
    if (!b) return;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    cudaFree(b->d_m);
    cudaFree(b->d_mid);
    cudaFree(b->d_aux);
    cudaFree(b->d_tile_e);
    cudaFree(b->d_E);
    cudaFree(b->d_slot_kT);
    cudaFree(b->d_noise_tab);
    cudaFree(b->d_reps);
    cudaFree(b->d_tiles);
    cudaFree(b->d_image);
    cudaFree(b->d_accept);
    cudaFree(b->d_stepctr);
    cudaFree(b->d_stage);
    cudaFree(b->d_gneb_part);
    cudaFree(b->d_mc_tiles);
    cudaFree(b->d_mc_acc);
    cudaFree(b->d_mc_prop);
    cudaFree(b->d_mc_cone);
    cudaFree(b->d_mc_cos);
    delete b;
}

// (re)build the tile list for the current variant and upload the replica table
mj_status batch_tiles(mj_batch* b, bool upload_reps) {
    const int ty = kBatchTY[b->variant];
    std::vector<int4> tiles;
    for (int r = 0; r < b->nrep; ++r) {
        BatchRep& R = b->reps[r];
        R.tile0 = static_cast<int>(tiles.size());
        for (int y0 = 0; y0 < R.Ly; y0 += ty)
            for (int x0 = 0; x0 < R.Lx; x0 += 32) tiles.push_back(make_int4(r, x0, y0, 0));
        R.ntiles = static_cast<int>(tiles.size()) - R.tile0;
    }
    b->ntile = static_cast<int>(tiles.size());
    cudaFree(b->d_tiles);
    cudaFree(b->d_tile_e);
    b->d_tiles = nullptr;
    b->d_tile_e = nullptr;
    mj_status st;
    if ((st = cuda_status(cudaMalloc(&b->d_tiles, sizeof(int4) * tiles.size()), "batch tiles")) != MJ_OK) return st;
    if ((st = cuda_status(cudaMalloc(&b->d_tile_e, sizeof(double) * tiles.size()), "batch tile energies")) != MJ_OK)
        return st;
    if ((st = cuda_status(cudaMemcpy(b->d_tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice),
                          "batch tiles")) != MJ_OK)
        return st;
    if (upload_reps)
        return cuda_status(cudaMemcpy(b->d_reps, b->reps.data(), sizeof(BatchRep) * b->nrep, cudaMemcpyHostToDevice),
                           "batch table");
    // keep the device table's temperatures (swaps), refresh only the tile ranges
    std::vector<BatchRep> cur(b->nrep);
    if ((st = cuda_status(cudaMemcpy(cur.data(), b->d_reps, sizeof(BatchRep) * b->nrep, cudaMemcpyDeviceToHost),
                          "batch table")) != MJ_OK)
        return st;
    for (int r = 0; r < b->nrep; ++r) {
        cur[r].tile0 = b->reps[r].tile0;
        cur[r].ntiles = b->reps[r].ntiles;
    }
    return cuda_status(cudaMemcpy(b->d_reps, cur.data(), sizeof(BatchRep) * b->nrep, cudaMemcpyHostToDevice),
                       "batch table");
}

mj_status batch_coef(const mj_batch* b, const mj_dyn_params* d, DynCoef& c, double& dt) {
    if (!d) return set_error(MJ_ERR_ARG, "null dynamics parameters");
    if (d->integrator != MJ_SIB) return set_error(MJ_ERR_UNSUPPORTED, "batches run the SIB integrator");
    if (!(d->timestep > 0.0) || !(d->alpha >= 0.0)) return set_error(MJ_ERR_ARG, "timestep must be > 0, alpha >= 0");
    if (d->noise == MJ_NOISE_INJECT) return set_error(MJ_ERR_UNSUPPORTED, "batches draw Philox noise or none");
    std::memset(&c, 0, sizeof(c));
    c.integrator = MJ_SIB;
    c.noise = d->noise;
    c.thermal = d->noise == MJ_NOISE_PHILOX && d->alpha > 0.0;
    c.alpha = d->alpha;
    c.inv_den = 1.0 / (1.0 + d->alpha * d->alpha);
    c.sib_hc = -0.5 * (d->timestep / kHbar) / (1.0 + d->alpha * d->alpha);
    c.seed = d->seed;
    c.stream_id = d->stream_id;  // replica r draws on stream_id + r
    uint32_t k0 = static_cast<uint32_t>(d->seed), k1 = static_cast<uint32_t>(d->seed >> 32);
    for (int r = 0; r < 10; ++r) {
        c.keys[2 * r] = k0;
        c.keys[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    c.noise_tab = b->d_noise_tab;
    c.step_base = nullptr;
    dt = d->timestep;  // sigma^2 = alpha kT hbar / dt per replica (dynamics/spindynamics.f90:266-272)
    return MJ_OK;
}

int batch_blocks(const mj_batch* b) {
    return std::max(1, std::min(b->ntile, b->num_sms * b->blocks_per_sm));
}

BatchArgs batch_args(mj_batch* b, uint32_t step, double dt) {
    BatchArgs A;
    A.reps = b->d_reps;
    A.tiles = b->d_tiles;
    A.ntile = b->ntile;
    A.Ntot = b->Ntot;
    A.ms = b->d_m;
    A.mn = b->d_m;
    A.out = b->d_mid;
    A.aux = b->d_aux;
    A.tile_e = nullptr;
    A.step = step;
    A.dt = dt;
    A.project = 0;
    A.tile_g = nullptr;
    A.gneb_n = 0;
    A.gneb_nimg = 0;
    return A;
}

mj_status batch_energy(mj_batch* b, const DynCoef& c, double* E, cudaStream_t s) {
    BatchArgs A = batch_args(b, 0, 0.0);
    A.tile_e = b->d_tile_e;
    mj_status st = batch_pass(b->shape, b->variant, BPASS_ENERGY, b->zaxial, b->sp, c, A, batch_blocks(b), s);
    if (st != MJ_OK) return st;
    k_batch_energy<<<b->nrep, 256, 0, s>>>(b->d_reps, b->nrep, b->d_tile_e, E);
    return cuda_status(cudaGetLastError(), "k_batch_energy");
}

// nsteps SIB steps; a PT round after every step whose global index + 1 is a multiple of swap_every
mj_status batch_sequence(mj_batch* b, const DynCoef& c0, double dt, uint32_t step0, int32_t nsteps,
                         int32_t swap_every, bool graph_mode, double* E_out, cudaStream_t s) {
    DynCoef c = c0;
    if (graph_mode) c.step_base = b->d_stepctr;
    mj_status st;
    const int nb = batch_blocks(b);
    for (int32_t k = 0; k < nsteps; ++k) {
        const uint32_t step = step0 + static_cast<uint32_t>(k);
        BatchArgs A = batch_args(b, step, dt);
        if ((st = batch_pass(b->shape, b->variant, BPASS_SIB1, b->zaxial, b->sp, c, A, nb, s)) != MJ_OK) return st;
        A.ms = b->d_mid;
        A.out = b->d_m;
        if ((st = batch_pass(b->shape, b->variant, BPASS_SIB2, b->zaxial, b->sp, c, A, nb, s)) != MJ_OK) return st;
        if (swap_every > 0 && ((step + 1) % static_cast<uint32_t>(swap_every)) == 0) {
            if ((st = batch_energy(b, c, b->d_E, s)) != MJ_OK) return st;
            // round index (step + 1) / swap_every; in a graph the device counter (a multiple of
            // swap_every) adds its share in the kernel
            const uint32_t round = (step + 1) / static_cast<uint32_t>(swap_every);
            k_pt_swap<<<1, 256, 0, s>>>(b->d_reps, b->d_image, b->d_slot_kT, b->nrep, b->d_E, c, round,
                                        static_cast<uint32_t>(swap_every), b->d_accept);
            if ((st = cuda_status(cudaGetLastError(), "k_pt_swap")) != MJ_OK) return st;
        }
    }
    if (E_out) return batch_energy(b, c, E_out, s);
    return MJ_OK;
}

// The field of the images for gneb_relax: the batch's field pass with the
// projection (BPASS_FIELD) and k_batch_energy; per iteration the GNEB field pass
// (projected fields and the path sums per tile) and k_gneb_img.
struct BatchFields {
    mj_batch* b;
    cudaStream_t s;
    double* tile_g;  // 6 path sums per tile
    DynCoef c;       // unused by the field passes (no dynamics)

    mj_status field(double* F, double* m, double* E) {
        BatchArgs A = batch_args(b, 0, 0.0);
        A.ms = A.mn = m;
        A.out = F;
        A.project = 1;
        A.tile_e = b->d_tile_e;
        mj_status e = batch_pass(b->shape, b->variant, BPASS_FIELD, b->zaxial, b->sp, c, A, batch_blocks(b), s);
        if (e != MJ_OK) return e;
        k_batch_energy<<<b->nrep, 256, 0, s>>>(b->d_reps, b->nrep, b->d_tile_e, E);
        return cuda_status(cudaGetLastError(), "k_batch_energy");
    }
    mj_status iterate(double* F, double* m, double* E, double* img, const GnebCtl* ctl) {
        BatchArgs A = batch_args(b, 0, 0.0);
        A.ms = A.mn = m;
        A.out = F;
        A.tile_e = b->d_tile_e;
        A.tile_g = tile_g;
        A.gneb_n = b->Ntot / b->nrep;
        A.gneb_nimg = b->nrep;
        mj_status e = batch_pass(b->shape, b->variant, BPASS_GNEB, b->zaxial, b->sp, c, A, batch_blocks(b), s);
        if (e != MJ_OK) return e;
        k_gneb_img<<<b->nrep, 256, 0, s>>>(b->d_reps, b->nrep, b->d_tile_e, tile_g, b->ntile, E, img, ctl);
        return cuda_status(cudaGetLastError(), "k_gneb_img");
    }
};

}  // namespace
}  // namespace mj

using namespace mj;

extern "C" {

mj_status mj_batch_create(const mj_lattice_desc* cell, const mj_hamiltonian_desc* ham, int32_t nrep, const int32_t* L,
                          const double* B_ext, const double* temperature, int32_t device, mj_batch** out) {
    if (!cell || !ham || !L || !B_ext || !temperature || !out || nrep < 1) return set_error(MJ_ERR_ARG, "bad batch arguments");
    *out = nullptr;
    if (ham->dip_on) return set_error(MJ_ERR_UNSUPPORTED, "batches do not carry the dipolar term");
    mj_status st = cuda_status(cudaSetDevice(device), "cudaSetDevice");
    if (st != MJ_OK) return st;
    int Lmax = 0;
    for (int r = 0; r < nrep; ++r) {
        if (L[2 * r] < 1 || L[2 * r + 1] < 1) return set_error(MJ_ERR_ARG, "replica sizes must be >= 1");
        Lmax = std::max(Lmax, std::max(L[2 * r], L[2 * r + 1]));
    }
    mj_lattice_desc lat = *cell;
    lat.L[0] = lat.L[1] = std::max(Lmax, 8);
    lat.L[2] = 1;
    Geometry g;
    std::string err;
    if (!build_geometry(lat, g, err)) return set_error(MJ_ERR_ARG, err);
    if (g.nmag != 1) return set_error(MJ_ERR_UNSUPPORTED, "batches need one magnetic atom per cell");
    std::vector<Block> blocks;
    std::vector<double> onsite;
    if (!build_blocks(g, *ham, blocks, onsite, err)) return set_error(MJ_ERR_GEOMETRY, err);
    mj_batch* b = new mj_batch();
    b->device = device;
    b->nrep = nrep;
    std::memset(&b->sp, 0, sizeof(b->sp));
    b->sp.periodic[0] = cell->periodic[0] ? 1 : 0;
    b->sp.periodic[1] = cell->periodic[1] ? 1 : 0;
    b->sp.L[0] = b->sp.L[1] = Lmax;
    b->sp.L[2] = 1;
    // the per-offset tensors are those of the single-lattice stencil
    if (!stencil_from_blocks(blocks, onsite, b->sp)) {
        batch_free(b);
        return set_error(MJ_ERR_UNSUPPORTED, "batches need a stencil lattice with a tiled shape");
    }
    match_shape(b->sp);
    b->shape = b->sp.shape;
    if (b->shape == kShapeGeneric) {
        batch_free(b);
        return set_error(MJ_ERR_UNSUPPORTED, "batches need a square or triangular lattice shape");
    }
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    const double zc = -((1.0 * kMuB * ham->c_zeeman) * cell->moment[g.magatom[0]]);
    b->L.assign(L, L + 2 * nrep);
    b->reps.resize(nrep);
    // temperature ladder: slots in ascending temperature, replica order breaks ties
    std::vector<int> order(nrep);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return temperature[a] < temperature[c]; });
    b->slot_kT.resize(nrep);
    std::vector<int> image(nrep);
    int64_t off = 0;
    bool zax = true;
    for (int r = 0; r < nrep; ++r) {
        BatchRep& R = b->reps[r];
        R.off = off;
        R.Lx = L[2 * r];
        R.Ly = L[2 * r + 1];
        off += static_cast<int64_t>(R.Lx) * R.Ly;
        // the Zeeman term is on when requested or when the field is not negligible (as for a plan)
        const double* Br = B_ext + 3 * r;
        const bool zee = ham->zeeman_on || std::sqrt(Br[0] * Br[0] + Br[1] * Br[1] + Br[2] * Br[2]) >= 1e-8;
        for (int k = 0; k < 3; ++k) R.zb[k] = zee ? zc * Br[k] : 0.0;
        if (R.zb[0] != 0.0 || R.zb[1] != 0.0) zax = false;
        R.kT = temperature[r] * kKB;
        R.stream = static_cast<uint32_t>(r);
    }
    b->zaxial = zax;
    for (int l = 0; l < nrep; ++l) {
        b->slot_kT[l] = temperature[order[l]] * kKB;
        image[l] = order[l];
        b->reps[order[l]].slot = l;
    }
    b->Ntot = off;
    auto dal = [&](auto** p, size_t n, const char* w) { return cuda_status(cudaMalloc(reinterpret_cast<void**>(p), n), w); };
    const size_t f3 = sizeof(double) * 3 * static_cast<size_t>(b->Ntot);
    if ((st = dal(&b->d_m, f3, "batch m")) != MJ_OK || (st = dal(&b->d_mid, f3, "batch mid")) != MJ_OK ||
        (st = dal(&b->d_aux, f3, "batch aux")) != MJ_OK || (st = dal(&b->d_E, sizeof(double) * nrep, "batch E")) != MJ_OK ||
        (st = dal(&b->d_slot_kT, sizeof(double) * nrep, "batch ladder")) != MJ_OK ||
        (st = dal(&b->d_noise_tab, sizeof(double) * kNoiseTabDoubles, "batch tables")) != MJ_OK ||
        (st = dal(&b->d_reps, sizeof(BatchRep) * nrep, "batch table")) != MJ_OK ||
        (st = dal(&b->d_image, sizeof(int) * nrep, "batch image")) != MJ_OK ||
        (st = dal(&b->d_accept, sizeof(int) * nrep, "batch accept")) != MJ_OK ||
        (st = dal(&b->d_stepctr, sizeof(uint32_t) * 4, "batch step counter")) != MJ_OK) {
        batch_free(b);
        return st;
    }
    {
        std::vector<double> tab(kNoiseTabDoubles);
        build_noise_tables(tab.data());
        cudaMemcpy(b->d_noise_tab, tab.data(), sizeof(double) * kNoiseTabDoubles, cudaMemcpyHostToDevice);
    }
    cudaMemcpy(b->d_slot_kT, b->slot_kT.data(), sizeof(double) * nrep, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_image, image.data(), sizeof(int) * nrep, cudaMemcpyHostToDevice);
    cudaMemset(b->d_accept, 0, sizeof(int) * nrep);
    cudaMemset(b->d_m, 0, f3);
    if ((st = batch_tiles(b, true)) != MJ_OK) {
        batch_free(b);
        return st;
    }
    if ((st = cuda_status(cudaDeviceSynchronize(), "batch create")) != MJ_OK) {
        batch_free(b);
        return st;
    }
    *out = b;
    return MJ_OK;
}

mj_status mj_batch_destroy(mj_batch* b) {
    if (!b) return MJ_OK;
    cudaSetDevice(b->device);
    batch_free(b);
    return MJ_OK;
}

mj_status mj_batch_nsites(const mj_batch* b, int64_t* total, int64_t* offsets) {
    if (!b || !total) return set_error(MJ_ERR_ARG, "null argument");
    *total = b->Ntot;
    if (offsets) {
        for (int r = 0; r < b->nrep; ++r) offsets[r] = b->reps[r].off;
        offsets[b->nrep] = b->Ntot;
    }
    return MJ_OK;
}

mj_status mj_batch_device_ptr(const mj_batch* b, double** m) {
    if (!b || !m) return set_error(MJ_ERR_ARG, "null argument");
    *m = b->d_m;
    return MJ_OK;
}

mj_status mj_batch_upload(mj_batch* b, const double* m, void* stream) {
    if (!b || !m) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(b->device);
    mj_status st;
    if (!b->d_stage && (st = cuda_status(cudaMalloc(&b->d_stage, sizeof(double) * 3 * b->Ntot), "batch stage")) != MJ_OK)
        return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((st = cuda_status(cudaMemcpyAsync(b->d_stage, m, sizeof(double) * 3 * b->Ntot, cudaMemcpyHostToDevice, s),
                          "batch upload")) != MJ_OK)
        return st;
    return aos_to_soa(b->d_stage, b->d_m, b->Ntot, s);
}

mj_status mj_batch_download(const mj_batch* bc, double* m, void* stream) {
    mj_batch* b = const_cast<mj_batch*>(bc);
    if (!b || !m) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(b->device);
    mj_status st;
    if (!b->d_stage && (st = cuda_status(cudaMalloc(&b->d_stage, sizeof(double) * 3 * b->Ntot), "batch stage")) != MJ_OK)
        return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((st = soa_to_aos(b->d_m, b->d_stage, b->Ntot, s)) != MJ_OK) return st;
    if ((st = cuda_status(cudaMemcpyAsync(m, b->d_stage, sizeof(double) * 3 * b->Ntot, cudaMemcpyDeviceToHost, s),
                          "batch download")) != MJ_OK)
        return st;
    return cuda_status(cudaStreamSynchronize(s), "batch download");
}

mj_status mj_batch_step(mj_batch* b, const mj_dyn_params* p, int32_t nsteps, int32_t swap_every, double* E_dev,
                        void* stream) {
    if (!b || nsteps < 0 || swap_every < 0) return set_error(MJ_ERR_ARG, "bad batch step arguments");
    cudaSetDevice(b->device);
    DynCoef c;
    double sc = 0.0;
    mj_status st = batch_coef(b, p, c, sc);
    if (st != MJ_OK) return st;
    return batch_sequence(b, c, sc, p->step0, nsteps, swap_every, false, E_dev, static_cast<cudaStream_t>(stream));
}

mj_status mj_batch_graph_run(mj_batch* b, const mj_dyn_params* p, int32_t steps_per_graph, int32_t nreplay,
                             int32_t swap_every, double* E_dev, void* stream) {
    if (!b || !p || steps_per_graph < 1 || nreplay < 0 || swap_every < 0)
        return set_error(MJ_ERR_ARG, "bad batch graph arguments");
    if (swap_every > 0 && steps_per_graph % swap_every != 0)
        return set_error(MJ_ERR_ARG, "steps_per_graph must be a multiple of swap_every");
    if (swap_every > 0 && p->step0 % static_cast<uint32_t>(swap_every) != 0)
        return set_error(MJ_ERR_ARG, "step0 must be a multiple of swap_every");
    cudaSetDevice(b->device);
    DynCoef c;
    double sc = 0.0;
    mj_status st = batch_coef(b, p, c, sc);
    if (st != MJ_OK) return st;
    if (!b->cap_stream &&
        (st = cuda_status(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking), "capture stream")) != MJ_OK)
        return st;
    std::string key(reinterpret_cast<const char*>(&c), sizeof(c));
    key += std::to_string(sc) + "/" + std::to_string(steps_per_graph) + "/" + std::to_string(swap_every) + "/" +
           std::to_string(reinterpret_cast<uintptr_t>(E_dev)) + "/" + std::to_string(b->variant) + "/" +
           std::to_string(b->blocks_per_sm);
    if (!b->graph || b->graph_key != key) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        cudaStream_t cs = b->cap_stream;
        if ((st = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture")) != MJ_OK)
            return st;
        mj_status inner = batch_sequence(b, c, sc, 0u, steps_per_graph, swap_every, true, E_dev, cs);
        if (inner == MJ_OK) inner = step_counter(b->d_stepctr, static_cast<uint32_t>(steps_per_graph), true, cs);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(cs, &graph);
        if (inner != MJ_OK) {
            if (graph) cudaGraphDestroy(graph);
            return inner;
        }
        if ((st = cuda_status(e, "end capture")) != MJ_OK) return st;
        e = cudaGraphInstantiate(&b->graph, graph, 0);
        cudaGraphDestroy(graph);
        if ((st = cuda_status(e, "graph instantiate")) != MJ_OK) {
            b->graph = nullptr;
            return st;
        }
        b->graph_key = key;
    }
    cudaStream_t us = static_cast<cudaStream_t>(stream);
    if ((st = step_counter(b->d_stepctr, p->step0, false, us)) != MJ_OK) return st;
    for (int32_t r = 0; r < nreplay; ++r)
        if ((st = cuda_status(cudaGraphLaunch(b->graph, us), "graph launch")) != MJ_OK) return st;
    return MJ_OK;
}

mj_status mj_batch_energies(mj_batch* b, double* E_host) {
    if (!b || !E_host) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(b->device);
    DynCoef c;
    std::memset(&c, 0, sizeof(c));
    mj_status st = batch_energy(b, c, b->d_E, 0);
    if (st != MJ_OK) return st;
    return cuda_status(cudaMemcpy(E_host, b->d_E, sizeof(double) * b->nrep, cudaMemcpyDeviceToHost), "batch energies");
}

mj_status mj_batch_temperatures(const mj_batch* b, double* T_host, int32_t* accepted) {
    if (!b || !T_host) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(b->device);
    std::vector<BatchRep> cur(b->nrep);
    mj_status st = cuda_status(cudaMemcpy(cur.data(), b->d_reps, sizeof(BatchRep) * b->nrep, cudaMemcpyDeviceToHost),
                               "batch table");
    if (st != MJ_OK) return st;
    for (int r = 0; r < b->nrep; ++r) T_host[r] = cur[r].kT / kKB;
    if (accepted)
        return cuda_status(cudaMemcpy(accepted, b->d_accept, sizeof(int) * b->nrep, cudaMemcpyDeviceToHost), "accepts");
    return MJ_OK;
}

mj_status mj_batch_field(mj_batch* b, double* B_dev, double* E_dev, int32_t project, void* stream) {
    if (!b || (!B_dev && !E_dev)) return set_error(MJ_ERR_ARG, "null argument");
    cudaSetDevice(b->device);
    DynCoef c;
    std::memset(&c, 0, sizeof(c));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BatchArgs A = batch_args(b, 0, 0.0);
    A.out = B_dev;
    A.project = project ? 1 : 0;
    A.tile_e = b->d_tile_e;
    mj_status st = batch_pass(b->shape, b->variant, B_dev ? BPASS_FIELD : BPASS_ENERGY, b->zaxial, b->sp, c, A, batch_blocks(b), s);
    if (st != MJ_OK) return st;
    if (E_dev) {
        k_batch_energy<<<b->nrep, 256, 0, s>>>(b->d_reps, b->nrep, b->d_tile_e, E_dev);
        return cuda_status(cudaGetLastError(), "k_batch_energy");
    }
    return MJ_OK;
}

mj_status mj_batch_gneb_tangent(mj_batch* b, const double* E_dev, int32_t mode, double* tau_dev, void* stream) {
    if (!b || !tau_dev || (mode == 0 && !E_dev) || mode < 0 || mode > 1) return set_error(MJ_ERR_ARG, "bad tangent arguments");
    for (int r = 1; r < b->nrep; ++r)
        if (b->reps[r].Lx != b->reps[0].Lx || b->reps[r].Ly != b->reps[0].Ly)
            return set_error(MJ_ERR_UNSUPPORTED, "path tangents need images of one size");
    cudaSetDevice(b->device);
    const int64_t n = b->Ntot / b->nrep;
    const int nblk = static_cast<int>((n + 255) / 256);
    mj_status st;
    if (!b->d_gneb_part &&
        (st = cuda_status(cudaMalloc(&b->d_gneb_part, sizeof(double) * nblk * b->nrep), "tangent partials")) != MJ_OK)
        return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const GnebIdx X{n, n, b->Ntot};
    k_gneb_tau<<<dim3(nblk, b->nrep), 256, 0, s>>>(b->d_m, X, b->nrep, E_dev, mode, tau_dev, b->d_gneb_part);
    if ((st = cuda_status(cudaGetLastError(), "k_gneb_tau")) != MJ_OK) return st;
    k_gneb_norm_sum<<<b->nrep, 256, 0, s>>>(b->d_gneb_part, nblk);
    k_gneb_scale<<<dim3(nblk, b->nrep), 256, 0, s>>>(tau_dev, X, b->d_gneb_part, nblk);
    return cuda_status(cudaGetLastError(), "k_gneb_scale");
}

mj_status mj_batch_set_config(mj_batch* b, int32_t variant, int32_t blocks_per_sm) {
    if (!b || variant < 0 || variant >= kBatchVariants || blocks_per_sm < 1 || blocks_per_sm > 64)
        return set_error(MJ_ERR_ARG, "variant 0..4 and blocks_per_sm 1..64");
    cudaSetDevice(b->device);
    const bool retile = variant != b->variant;
    b->variant = variant;
    b->blocks_per_sm = blocks_per_sm;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        b->graph_key.clear();
    }
    return retile ? batch_tiles(b, false) : MJ_OK;
}

mj_status mj_batch_autotune(mj_batch* b, const mj_dyn_params* p, int32_t steps, int32_t* best_variant,
                            int32_t* best_bps, double* ms_table) {
    if (!b || !p || steps < 1 || !best_variant || !best_bps) return set_error(MJ_ERR_ARG, "bad autotune arguments");
    cudaSetDevice(b->device);
    DynCoef c;
    double sc = 0.0;
    mj_status st = batch_coef(b, p, c, sc);
    if (st != MJ_OK) return st;
    // time on a copy of the state; the table's temperatures are not swapped here
    double* save = nullptr;
    if ((st = cuda_status(cudaMalloc(&save, sizeof(double) * 3 * b->Ntot), "autotune copy")) != MJ_OK) return st;
    cudaMemcpy(save, b->d_m, sizeof(double) * 3 * b->Ntot, cudaMemcpyDeviceToDevice);
    static const int bps_list[5] = {2, 4, 8, 16, 32};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int bv = b->variant, bb = b->blocks_per_sm;
    int k = 0;
    for (int v = 0; v < kBatchVariants && st == MJ_OK; ++v)
        for (int q = 0; q < 5 && st == MJ_OK; ++q, ++k) {
            if ((st = mj_batch_set_config(b, v, bps_list[q])) != MJ_OK) break;
            if ((st = batch_sequence(b, c, sc, p->step0, 1, 0, false, nullptr, 0)) != MJ_OK) break;
            cudaEventRecord(e0, 0);
            if ((st = batch_sequence(b, c, sc, p->step0, steps, 0, false, nullptr, 0)) != MJ_OK) break;
            cudaEventRecord(e1, 0);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double per = ms / steps;
            if (ms_table) ms_table[k] = per;
            if (per < best) {
                best = per;
                bv = v;
                bb = bps_list[q];
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemcpy(b->d_m, save, sizeof(double) * 3 * b->Ntot, cudaMemcpyDeviceToDevice);
    cudaFree(save);
    if (st != MJ_OK) return st;
    if ((st = mj_batch_set_config(b, bv, bb)) != MJ_OK) return st;
    *best_variant = bv;
    *best_bps = bb;
    return cuda_status(cudaDeviceSynchronize(), "batch autotune");
}

// ---- Monte Carlo on the replicas -------------------------------------------

// the colouring of every replica, its MC tile list and the per-replica chain state (first call)
static mj_status batch_mc_setup(mj_batch* b, double cone0, cudaStream_t s) {
    if (b->d_mc_tiles) return MJ_OK;
    std::vector<int> L3(3 * b->nrep);
    for (int r = 0; r < b->nrep; ++r) {
        L3[3 * r] = b->reps[r].Lx;
        L3[3 * r + 1] = b->reps[r].Ly;
        L3[3 * r + 2] = 1;
    }
    if (!mc_colouring(b->sp, L3.data(), b->nrep, b->mc_col))
        return set_error(MJ_ERR_UNSUPPORTED, "no linear or product colouring fits the stencil and every "
                                             "replica's sizes");
    const McClass K0 = mc_classes(b->mc_col)[0];
    std::vector<int4> tiles;
    for (int r = 0; r < b->nrep; ++r) {
        const int nx = (b->reps[r].Lx + K0.qx - 1) / K0.qx, ny = (b->reps[r].Ly + K0.sy - 1) / K0.sy;
        for (int by = 0; by < (ny + kMcBY - 1) / kMcBY; ++by)
            for (int bx = 0; bx < (nx + 31) / 32; ++bx) tiles.push_back(make_int4(r, bx, by, 0));
    }
    b->mc_ntile = static_cast<int>(tiles.size());
    const int nrep = b->nrep;
    mj_status st;
    if ((st = cuda_status(cudaMalloc(&b->d_mc_tiles, sizeof(int4) * tiles.size()), "MC tiles")) != MJ_OK ||
        (st = cuda_status(cudaMalloc(&b->d_mc_acc, sizeof(unsigned long long) * nrep), "MC state")) != MJ_OK ||
        (st = cuda_status(cudaMalloc(&b->d_mc_prop, sizeof(long long) * nrep), "MC state")) != MJ_OK ||
        (st = cuda_status(cudaMalloc(&b->d_mc_cone, sizeof(double) * nrep), "MC state")) != MJ_OK ||
        (st = cuda_status(cudaMalloc(&b->d_mc_cos, sizeof(double) * nrep), "MC state")) != MJ_OK) {
        cudaFree(b->d_mc_tiles);
        b->d_mc_tiles = nullptr;
        return st;
    }
    if ((st = cuda_status(cudaMemcpy(b->d_mc_tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice),
                          "MC tiles")) != MJ_OK)
        return st;
    k_batch_mc_init<<<(nrep + 127) / 128, 128, 0, s>>>(nrep, cone0, b->d_mc_acc, b->d_mc_prop, b->d_mc_cone,
                                                       b->d_mc_cos);
    return cuda_status(cudaGetLastError(), "k_batch_mc_init");
}

mj_status mj_batch_mc_reset(mj_batch* b, double cone) {
    if (!b || !(cone > 0.0)) return set_error(MJ_ERR_ARG, "bad batch Monte Carlo reset");
    cudaSetDevice(b->device);
    mj_status st = batch_mc_setup(b, cone, 0);
    if (st != MJ_OK) return st;
    k_batch_mc_init<<<(b->nrep + 127) / 128, 128>>>(b->nrep, cone, b->d_mc_acc, b->d_mc_prop, b->d_mc_cone,
                                                    b->d_mc_cos);
    if ((st = cuda_status(cudaGetLastError(), "k_batch_mc_init")) != MJ_OK) return st;
    return cuda_status(cudaDeviceSynchronize(), "batch Monte Carlo reset");
}

mj_status mj_batch_mc(mj_batch* b, mj_mc_params* p, int32_t nrounds, int32_t sweeps_per_round, int32_t swap,
                      double* E_dev, double* M_dev, int32_t* slot_dev, int32_t* colors, void* stream) {
    if (!b || !p || nrounds < 0 || sweeps_per_round < 1) return set_error(MJ_ERR_ARG, "bad batch Monte Carlo arguments");
    if (p->proposal < MJ_MC_CONE || p->proposal > MJ_MC_OVERRELAX) return set_error(MJ_ERR_ARG, "unknown proposal");
    if (!(p->cone > 0.0)) return set_error(MJ_ERR_ARG, "cone > 0");
    cudaSetDevice(b->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    mj_status st = batch_mc_setup(b, p->cone, s);
    if (st != MJ_OK) return st;
    if (colors)
        for (int d = 0; d < 4; ++d) colors[d] = b->mc_col[d];
    const std::vector<McClass> classes = mc_classes(b->mc_col);
    BatchMcArgs A;
    std::memset(&A, 0, sizeof(A));
    A.tab = b->d_noise_tab;
    A.reps = b->d_reps;
    A.tiles = b->d_mc_tiles;
    A.Ntot = b->Ntot;
    A.m = b->d_m;
    A.cos_cone = b->d_mc_cos;
    A.acc = b->d_mc_acc;
    mc_keys(p->seed, A.keys);
    A.proposal = p->proposal;
    A.stream_id = p->stream_id;
    DynCoef c;  // the swap test's Philox key (no device step counter)
    std::memset(&c, 0, sizeof(c));
    mc_keys(p->seed, c.keys);
    const int adapt = p->adapt_cone && p->proposal == MJ_MC_CONE;
    const int nrep = b->nrep;
    for (int32_t k = 0; k < nrounds; ++k) {
        for (int32_t t = 0; t < sweeps_per_round; ++t) {
            A.sweep = p->sweep0 + static_cast<uint32_t>(k * sweeps_per_round + t);
            for (const McClass& K : classes) {
                A.K = K;
                switch (b->shape) {
                    case kShapeSquareNN: k_batch_mc<ShapeSquareNN><<<b->mc_ntile, dim3(32, kMcBY), 0, s>>>(b->sp, A); break;
                    case kShapeSquare2: k_batch_mc<ShapeSquare2><<<b->mc_ntile, dim3(32, kMcBY), 0, s>>>(b->sp, A); break;
                    case kShapeTriNN: k_batch_mc<ShapeTriNN><<<b->mc_ntile, dim3(32, kMcBY), 0, s>>>(b->sp, A); break;
                    case kShapeTri3: k_batch_mc<ShapeTri3><<<b->mc_ntile, dim3(32, kMcBY), 0, s>>>(b->sp, A); break;
                    default: k_batch_mc<void><<<b->mc_ntile, dim3(32, kMcBY), 0, s>>>(b->sp, A);
                }
            }
            k_batch_mc_cone<<<(nrep + 127) / 128, 128, 0, s>>>(b->d_reps, nrep, b->d_mc_acc, b->d_mc_prop,
                                                               b->d_mc_cone, b->d_mc_cos, adapt);
            if ((st = cuda_status(cudaGetLastError(), "k_batch_mc")) != MJ_OK) return st;
        }
        // measure (measure_add) before the swap, with the temperatures the sweeps had
        double* E = E_dev ? E_dev + static_cast<int64_t>(k) * nrep : b->d_E;
        if ((E_dev || swap) && (st = batch_energy(b, c, E, s)) != MJ_OK) return st;
        if (M_dev || slot_dev) {
            k_batch_magnet<<<nrep, 256, 0, s>>>(b->d_reps, b->d_m, b->Ntot,
                                                M_dev ? M_dev + 3 * static_cast<int64_t>(k) * nrep : nullptr,
                                                slot_dev ? slot_dev + static_cast<int64_t>(k) * nrep : nullptr);
            if ((st = cuda_status(cudaGetLastError(), "k_batch_magnet")) != MJ_OK) return st;
        }
        if (swap) {
            k_pt_swap<<<1, 256, 0, s>>>(b->d_reps, b->d_image, b->d_slot_kT, nrep, E, c, p->round0 + static_cast<uint32_t>(k),
                                        1u, b->d_accept);
            if ((st = cuda_status(cudaGetLastError(), "k_pt_swap")) != MJ_OK) return st;
        }
    }
    p->sweep0 += static_cast<uint32_t>(nrounds * sweeps_per_round);
    if (swap) p->round0 += static_cast<uint32_t>(nrounds);
    return MJ_OK;
}

mj_status mj_batch_mc_state(mj_batch* b, double* cone, int64_t* accepted, int64_t* proposed) {
    if (!b) return set_error(MJ_ERR_ARG, "null batch");
    if (!b->d_mc_tiles) return set_error(MJ_ERR_ARG, "no Monte Carlo has run on this batch");
    cudaSetDevice(b->device);
    mj_status st = cuda_status(cudaDeviceSynchronize(), "batch Monte Carlo");
    const size_t n = static_cast<size_t>(b->nrep);
    if (st == MJ_OK && cone) st = cuda_status(cudaMemcpy(cone, b->d_mc_cone, sizeof(double) * n, cudaMemcpyDeviceToHost), "MC state");
    if (st == MJ_OK && accepted)
        st = cuda_status(cudaMemcpy(accepted, b->d_mc_acc, sizeof(int64_t) * n, cudaMemcpyDeviceToHost), "MC state");
    if (st == MJ_OK && proposed)
        st = cuda_status(cudaMemcpy(proposed, b->d_mc_prop, sizeof(int64_t) * n, cudaMemcpyDeviceToHost), "MC state");
    return st;
}

// ---- GNEB path relaxation --------------------------------------------------

mj_status mj_batch_gneb_path(mj_batch* b, const mj_gneb_params* p, double* rx, double* ene, double* dene,
                             int64_t* iterations, double* max_force, int32_t* climbing) {
    if (!b) return set_error(MJ_ERR_ARG, "bad GNEB arguments (no batch)");
    mj_status st = gneb_check(p, b->nrep, rx, ene, dene);
    if (st != MJ_OK) return st;
    for (int r = 1; r < b->nrep; ++r)
        if (b->reps[r].Lx != b->reps[0].Lx || b->reps[r].Ly != b->reps[0].Ly)
            return set_error(MJ_ERR_UNSUPPORTED, "a path needs images of one size");
    cudaSetDevice(b->device);
    const int nrep = b->nrep;
    const int64_t Ntot = b->Ntot, n = Ntot / nrep;
    if (!b->cap_stream &&
        (st = cuda_status(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking), "capture stream")) != MJ_OK)
        return st;
    BatchFields fl{b, b->cap_stream, nullptr, DynCoef{}};
    std::memset(&fl.c, 0, sizeof(fl.c));
    if ((st = cuda_status(cudaMalloc(&fl.tile_g, sizeof(double) * 6 * b->ntile), "GNEB buffers")) != MJ_OK) return st;
    // the path as the work queued on the legacy default stream (an upload) leaves it
    st = cuda_status(cudaStreamSynchronize(0), "GNEB start");
    if (st == MJ_OK)
        st = gneb_relax(fl, b->d_m, nrep, GnebIdx{n, n, Ntot}, b->num_sms, b->cap_stream, p, 32, rx, ene, dene,
                        iterations, max_force, climbing);
    cudaFree(fl.tile_g);
    return st;
}

}  // extern "C"
