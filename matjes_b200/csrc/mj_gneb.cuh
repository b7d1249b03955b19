// GNEB path relaxation: find_path of GNEB/gneb_utils.f90:19-240 on the device,
// shared by the two holders of a path.  A path of nrep images of n sites is one
// device array; GnebIdx says where site li of image r is (index r is + li) and
// how far apart its three components are (cs):
//   a replica batch (images = replicas, x[Ntot] | y[Ntot] | z[Ntot]): is = n, cs = Ntot;
//   a plan's lattice (image r the SoA block [3n] at 3 n r):           is = 3n, cs = n.
// The caller supplies the field of the images (a Fields object):
//   field(F, m, E):             projected fields and energies of the spins m;
//   iterate(F, m, E, img, ctl): the same and the six path sums of every image
//                               (|A|^2, A.B, |B|^2, F.A, F.B, squared angle to
//                               image r + 1, at img[q nrep + r]; A = P(m_{r+1} - m),
//                               B = P(m - m_{r-1}), zero at the path's ends).
// An iteration is that, k_gneb_step (GNEB force, transport, velocity Verlet,
// velocity projection, stop flag) and k_gneb_move; chunks of iterations replay
// as one CUDA graph.  Every sum is a block partial summed in a fixed order, so
// the iterations are deterministic.  Included by mj_batch.cu and mj_gneb.cu;
// everything here has internal linkage.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "mj_device.cuh"

namespace mj {
namespace {

struct GnebIdx {
    int64_t n;   // sites of an image
    int64_t is;  // image stride: site li of image r at r is + li
    int64_t cs;  // component stride
};

// GNEB path tangents (GNEB/tangent.f90): for image r with neighbours r-1, r+1
// tau = wp (m_{r+1} - m_r) + wm (m_r - m_{r-1}), projected on the tangent space
// of m_r (vec_project, vector_utils/vector.f90:61-72) and normalised over the
// image.  mode 0 (lattice_special, :93-124, doi:10.1016/j.cpc.2015.07.001):
// the energy-weighted tangent of interior images; mode 1 (lattice_single,
// :163-180): m_{r+1} - m_{r-1}.  End images take the one-sided difference.
__device__ __forceinline__ void gneb_weights(const double* E, int r, int nrep, int mode, double& wp, double& wm) {
    if (r == 0) {
        wp = 1.0;
        wm = 0.0;
        return;
    }
    if (r == nrep - 1) {
        wp = 0.0;
        wm = 1.0;
        return;
    }
    if (mode == 1) {
        wp = wm = 1.0;
        return;
    }
    const double u1 = E[r - 1], u2 = E[r], u3 = E[r + 1];
    if (u3 > u2 && u2 > u1) {
        wp = 1.0;
        wm = 0.0;
    } else if (u1 > u2 && u2 > u3) {
        wp = 0.0;
        wm = 1.0;
    } else {
        double dmax = fabs(u3 - u2), dmin = fabs(u1 - u2);
        if (dmax < dmin) {
            const double t = dmax;
            dmax = dmin;
            dmin = t;
        }
        if (u3 > u1) {
            wp = dmax;
            wm = dmin;
        } else {
            wp = dmin;
            wm = dmax;
        }
    }
}

// unnormalised projected tangents; partial |tau|^2 per (image, block)
__global__ void __launch_bounds__(256) k_gneb_tau(const double* __restrict__ m, GnebIdx X, int nrep,
                                                  const double* __restrict__ E, int mode, double* __restrict__ tau,
                                                  double* __restrict__ part) {
    const int r = blockIdx.y;
    const int64_t li = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double wp, wm;
    gneb_weights(E, r, nrep, mode, wp, wm);
    double q = 0.0;
    if (li < X.n) {
        const int64_t i = r * X.is + li;
        const double3 m0 = ld3(m, i, X.cs);
        const double3 mp = r + 1 < nrep ? ld3(m, i + X.is, X.cs) : m0;
        const double3 mm = r > 0 ? ld3(m, i - X.is, X.cs) : m0;
        double3 t = make_double3(wp * (mp.x - m0.x) + wm * (m0.x - mm.x), wp * (mp.y - m0.y) + wm * (m0.y - mm.y),
                                 wp * (mp.z - m0.z) + wm * (m0.z - mm.z));
        const double d = dot(t, m0);
        t = make_double3(t.x - d * m0.x, t.y - d * m0.y, t.z - d * m0.z);
        st3(tau, i, X.cs, t);
        q = dot(t, t);
    }
    double v[1] = {q};
    block_partials<1>(v, part + static_cast<int64_t>(r) * gridDim.x, gridDim.x, blockIdx.x);
}

// per image: the ordered sum of its partials; 1/sqrt(sum) left in the image's
// first partial
__global__ void __launch_bounds__(256) k_gneb_norm_sum(double* part, int nblk) {
    const int r = blockIdx.x;
    __shared__ double tot;
    ordered_sum<1>(part + static_cast<int64_t>(r) * nblk, nblk, &tot);
    __syncthreads();
    if (threadIdx.x == 0) part[static_cast<int64_t>(r) * nblk] = tot > 0.0 ? 1.0 / sqrt(tot) : 0.0;
}

// tau /= |tau| of its image
__global__ void __launch_bounds__(256) k_gneb_scale(double* __restrict__ tau, GnebIdx X,
                                                    const double* __restrict__ part, int nblk) {
    const int r = blockIdx.y;
    const int64_t li = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (li >= X.n) return;
    const double inv = part[static_cast<int64_t>(r) * nblk];
    const int64_t i = r * X.is + li;
    tau[i] *= inv;
    tau[X.cs + i] *= inv;
    tau[2 * X.cs + i] *= inv;
}

__device__ __forceinline__ double3 gneb_rotate(double3 v, double3 a, double sn, double cs) {
    // utilities/rotation.f90 rotate_vector_arr: v cos + sin (v x a) + (1 - cos)(a.v) a
    const double t = dot(a, v);
    return make_double3(v.x * cs + sn * (a.z * v.y - a.y * v.z) + (1.0 - cs) * t * a.x,
                        v.y * cs + sn * (a.x * v.z - a.z * v.x) + (1.0 - cs) * t * a.y,
                        v.z * cs + sn * (a.y * v.x - a.x * v.y) + (1.0 - cs) * t * a.z);
}
__device__ __forceinline__ double gneb_ang(double3 a, double3 b) {
    const double3 c = cross(a, b);
    return atan2(sqrt(dot(c, c)), dot(a, b));
}

// partial sums of the squared spin angles between images r and r + 1 (the_path)
__global__ void __launch_bounds__(256) k_gneb_seg(const double* __restrict__ m, GnebIdx X, double* part) {
    const int r = blockIdx.y;
    const int64_t li = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double v[1] = {0.0};
    if (li < X.n) {
        const int64_t i = r * X.is + li;
        const double l = gneb_ang(ld3(m, i, X.cs), ld3(m, i + X.is, X.cs));
        v[0] = l * l;
    }
    block_partials<1>(v, part + static_cast<int64_t>(r) * gridDim.x, gridDim.x, blockIdx.x);
}

__global__ void __launch_bounds__(256) k_gneb_pathlen(const double* part, int nblk, int nrep, double* pl) {
    __shared__ double seg;
    if (threadIdx.x == 0) pl[0] = 0.0;
    for (int r = 0; r + 1 < nrep; ++r) {
        ordered_sum<1>(part + static_cast<int64_t>(r) * nblk, nblk, &seg);
        __syncthreads();
        if (threadIdx.x == 0) pl[r + 1] = pl[r] + sqrt(seg);
        __syncthreads();
    }
}

// partial sums of a.b per image
__global__ void __launch_bounds__(256) k_gneb_dot(const double* __restrict__ a, const double* __restrict__ b, GnebIdx X,
                                                  double* part) {
    const int r = blockIdx.y;
    const int64_t li = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double v[1] = {0.0};
    if (li < X.n) {
        const int64_t i = r * X.is + li;
        v[0] = dot(ld3(a, i, X.cs), ld3(b, i, X.cs));
    }
    block_partials<1>(v, part + static_cast<int64_t>(r) * gridDim.x, gridDim.x, blockIdx.x);
}

// per image: the ordered sum of its partials
__global__ void __launch_bounds__(256) k_gneb_dot_img(const double* part, int nblk, double* out) {
    ordered_sum<1>(part + static_cast<int64_t>(blockIdx.x) * nblk, nblk, out + blockIdx.x);
}

// maxloc of the image energies: the first image of highest energy (the climbing
// image, gneb_utils.f90:84,159)
__device__ __forceinline__ int gneb_maxloc(const double* E, int nrep) {
    int c = 0;
    for (int q = 1; q < nrep; ++q)
        if (E[q] > E[c]) c = q;
    return c;
}

// interior: F = F - tau (F.tau) + k (l_{r+1} + l_{r-1} - 2 l_r) tau, at the
// climbing image (climb != 0) F - 2 tau (F.tau); end images: 0, or left as they
// are (keep_ends, the forces before the first move)
__global__ void __launch_bounds__(256) k_gneb_force(double* F, const double* __restrict__ tau, const double* __restrict__ fp,
                                                    const double* __restrict__ pl, const double* __restrict__ E,
                                                    GnebIdx X, int nrep, double spring, int keep_ends, int climb) {
    const int r = blockIdx.y;
    const int64_t li = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (li >= X.n) return;
    const int64_t i = r * X.is + li;
    if (r == 0 || r == nrep - 1) {
        if (!keep_ends) st3(F, i, X.cs, make_double3(0.0, 0.0, 0.0));
        return;
    }
    const double3 f = ld3(F, i, X.cs), t = ld3(tau, i, X.cs);
    if (climb && gneb_maxloc(E, nrep) == r) {
        const double a2 = 2.0 * fp[r];
        st3(F, i, X.cs, make_double3(f.x - t.x * a2, f.y - t.y * a2, f.z - t.z * a2));
        return;
    }
    const double a = fp[r], k = spring * (pl[r + 1] + pl[r - 1] - 2.0 * pl[r]);
    st3(F, i, X.cs, make_double3(f.x - t.x * a + k * t.x, f.y - t.y * a + k * t.y, f.z - t.z * a + k * t.z));
}

// one partial max |F| per block over a flat array (the forces before the first move)
__global__ void __launch_bounds__(256) k_gneb_absmax(const double* __restrict__ F, int64_t n3, double* pmax) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double fm = k < n3 ? fabs(F[k]) : 0.0;
    __shared__ double wmax[8];
    for (int o = 16; o > 0; o >>= 1) fm = fmax(fm, __shfl_down_sync(0xffffffffu, fm, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = fm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x) / 32; ++w) mx = fmax(mx, wmax[w]);
        pmax[blockIdx.x] = mx;
    }
}

__global__ void __launch_bounds__(256) k_gneb_maxof(const double* __restrict__ pmax, int nb, double* out) {
    double fm = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) fm = fmax(fm, pmax[b]);
    __shared__ double wmax[8];
    for (int o = 16; o > 0; o >>= 1) fm = fmax(fm, __shfl_down_sync(0xffffffffu, fm, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = fm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x) / 32; ++w) mx = fmax(mx, wmax[w]);
        *out = mx;
    }
}

// F -= (F.m) m (project, vector_utils/vector.f90:61-72)
__global__ void __launch_bounds__(256) k_gneb_project(double* F, const double* __restrict__ m, GnebIdx X) {
    const int r = blockIdx.y;
    const int64_t li = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (li >= X.n) return;
    const int64_t i = r * X.is + li;
    const double3 f = ld3(F, i, X.cs), m0 = ld3(m, i, X.cs);
    const double d = dot(f, m0);
    st3(F, i, X.cs, make_double3(f.x - d * m0.x, f.y - d * m0.y, f.z - d * m0.z));
}

// Iteration state on the device: done set by the iteration that stopped (max |F|
// < ftol or itrmax reached; the iterations after it in a graph do no work but
// the field pass); the iterations taken.
struct GnebCtl {
    int done;
    int pad;
    long long iters;
};

// The energy-weighted tangent of image r at site i (unnormalised, projected on
// the spin: lattice_special, GNEB/tangent.f90:93-124); m0, mp its spin and the
// next image's.
__device__ __forceinline__ double3 gneb_tangent_site(const double* __restrict__ m, int64_t i, const GnebIdx& X, int r,
                                                     int nrep, double wp, double wm, double3& m0, double3& mp) {
    m0 = ld3(m, i, X.cs);
    mp = r + 1 < nrep ? ld3(m, i + X.is, X.cs) : m0;
    const double3 mm = r > 0 ? ld3(m, i - X.is, X.cs) : m0;
    double3 t = make_double3(wp * (mp.x - m0.x) + wm * (m0.x - mm.x), wp * (mp.y - m0.y) + wm * (m0.y - mm.y),
                             wp * (mp.z - m0.z) + wm * (m0.z - mm.z));
    const double d = dot(t, m0);
    return make_double3(t.x - d * m0.x, t.y - d * m0.y, t.z - d * m0.z);
}


// Per image (r = blockIdx.x): F projected in place and the six path sums; the
// last block of an image sums the partials in block order into img[q nrep + r].
// With esite (per-site energies, image r at esite[r n, (r + 1) n)) also their
// sum into E[r].  For fields that come without them (a plan's field kernels);
// ctl may be null (always runs).  SPT sites per thread, 256 apart (coalesced),
// so that the seven block reductions are paid once per SPT sites.
template <int SPT>
__global__ void __launch_bounds__(256) k_gneb_sums(const double* __restrict__ m, double* F, GnebIdx X, int nrep,
                                                   const double* __restrict__ esite, double* E, double* part,
                                                   unsigned int* cnt, double* img, const GnebCtl* ctl) {
    if (ctl && ctl->done) return;
    const int r = blockIdx.x;
    const int nblk = gridDim.y;
    double g[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const bool up = r + 1 < nrep;
#pragma unroll
    for (int q = 0; q < SPT; ++q) {
        const int64_t li = (blockIdx.y * static_cast<int64_t>(SPT) + q) * blockDim.x + threadIdx.x;
        if (li < X.n) {
            const int64_t i = r * X.is + li;
            const double3 m0 = ld3(m, i, X.cs);
            const double3 mp = up ? ld3(m, i + X.is, X.cs) : m0;
            const double3 mm = r > 0 ? ld3(m, i - X.is, X.cs) : m0;
            double3 f = ld3(F, i, X.cs);
            const double d = dot(f, m0);
            f = make_double3(f.x - d * m0.x, f.y - d * m0.y, f.z - d * m0.z);
            st3(F, i, X.cs, f);
            double g6[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            gneb_path_terms(m0, mp, mm, up, f, g6);
            for (int k = 0; k < 6; ++k) g[k] += g6[k];
            if (esite) g[6] += esite[r * X.n + li];
        }
    }
    double* pr = part + static_cast<int64_t>(r) * 7 * nblk;
    block_partials<7>(g, pr, nblk, blockIdx.y);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(cnt + r, 1u) == static_cast<unsigned int>(nblk - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double sums[7];
    ordered_sum<7>(pr, nblk, sums);
    if (threadIdx.x == 0) {
        for (int q = 0; q < 6; ++q) img[q * nrep + r] = sums[q];
        if (esite) E[r] = sums[6];
        cnt[r] = 0u;
    }
}

// Interior images: tau = wp A + wm B (the energy-weighted tangent at the site,
// the weights of the image energies) over |tau| from the image's path sums, F =
// F - tau (F.tau) + k (seg_r - seg_{r-1}) tau, stored; the old velocity lam Fo
// (the projection of the previous iteration, lam = scal[3]) and the old force Fo
// carried along the rotation R that took the spin from mo to m, v = lam R Fo +
// (R Fo + F) dt / (2 mass).  At the climbing image (climb) F - 2 tau (F.tau)
// instead.  End images: F = v = 0.  The last block sums v.F and F.F in block
// order, takes max |F|, sets lam = v.F / F.F (0 when v.F < 0; the velocity
// projection, v = lam F), counts the iteration and sets the stop flag.  r =
// blockIdx.x: the images of one site range run side by side, so the
// neighbouring images' spins come from L2.
template <int SPT>
__global__ void __launch_bounds__(256, 4) k_gneb_step(const double* __restrict__ m, const double* __restrict__ mo,
                                                   const double* __restrict__ Fo, double* Fn,
                                                   const double* __restrict__ E, const double* __restrict__ img,
                                                   GnebIdx X, int nrep, double spring, double dt, double mass,
                                                   double ftol, long long itrmax, int climb, double* part,
                                                   double* pmax, unsigned int* cnt, GnebCtl* ctl, double* scal) {
    if (ctl->done) return;
    const int r = blockIdx.x;
    const int nb = gridDim.x * gridDim.y, bid = blockIdx.x + gridDim.x * blockIdx.y;
    const bool inner = r > 0 && r < nrep - 1;
    double wp = 0.0, wm = 0.0, inv = 0.0, a = 0.0, k = 0.0;
    if (inner) {
        gneb_weights(E, r, nrep, 0, wp, wm);
        const double t2 = wp * wp * img[r] + 2.0 * wp * wm * img[nrep + r] + wm * wm * img[2 * nrep + r];
        inv = t2 > 0.0 ? 1.0 / sqrt(t2) : 0.0;
        a = (wp * img[3 * nrep + r] + wm * img[4 * nrep + r]) * inv;
        k = spring * (sqrt(img[5 * nrep + r]) - sqrt(img[5 * nrep + r - 1]));
        if (climb) {
            __shared__ int ci_s;
            if (threadIdx.x == 0) ci_s = gneb_maxloc(E, nrep);
            __syncthreads();
            if (ci_s == r) {
                // the climbing image: F - 2 tau (F.tau), no spring
                a *= 2.0;
                k = 0.0;
            }
        }
    }
    const double h = 0.5 / mass * dt, lam = scal[3];
    double v2[2] = {0.0, 0.0}, fm = 0.0;
#pragma unroll
    for (int q = 0; q < SPT; ++q) {
        const int64_t li = (static_cast<int64_t>(blockIdx.y) * SPT + q) * blockDim.x + threadIdx.x;
        if (li >= X.n) break;
        const int64_t i = r * X.is + li;
        double3 f = make_double3(0.0, 0.0, 0.0), v = f;
        if (inner) {
            double3 m0, mp;
            const double3 t0 = gneb_tangent_site(m, i, X, r, nrep, wp, wm, m0, mp);
            const double3 t = make_double3(t0.x * inv, t0.y * inv, t0.z * inv);
            const double3 g = ld3(Fn, i, X.cs);
            f = make_double3(g.x - t.x * a + k * t.x, g.y - t.y * a + k * t.y, g.z - t.z * a + k * t.z);
            // the move's rotation: axis mo x Fo/|Fo| (rotation_axis_arr), angle
            // between mo and m (sin |m x mo|, cos m.mo)
            const double3 m1 = ld3(mo, i, X.cs), fo = ld3(Fo, i, X.cs);
            double3 fn = fo;
            const double nf = sqrt(dot(fo, fo));
            if (nf > 1e-30) fn = make_double3(fo.x / nf, fo.y / nf, fo.z / nf);
            double3 e = cross(m1, fn);
            const double ne = sqrt(dot(e, e));
            if (ne > 2.220446049250313e-16) e = make_double3(e.x / ne, e.y / ne, e.z / ne);
            const double3 c = cross(m0, m1);
            const double3 fr = gneb_rotate(fo, e, sqrt(dot(c, c)), dot(m0, m1));
            v = make_double3(lam * fr.x + (fr.x + f.x) * h, lam * fr.y + (fr.y + f.y) * h,
                             lam * fr.z + (fr.z + f.z) * h);
        }
        st3(Fn, i, X.cs, f);
        v2[0] += dot(v, f);
        v2[1] += dot(f, f);
        fm = fmax(fm, fmax(fabs(f.x), fmax(fabs(f.y), fabs(f.z))));
    }
    block_partials<2>(v2, part, nb, bid);
    __shared__ double wmax[8];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) fm = fmax(fm, __shfl_down_sync(0xffffffffu, fm, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = fm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x) / 32; ++w) mx = fmax(mx, wmax[w]);
        pmax[bid] = mx;
        __threadfence();
        last = atomicAdd(cnt, 1u) == static_cast<unsigned int>(nb - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double sums[2];
    ordered_sum<2>(part, nb, sums);
    fm = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) fm = fmax(fm, __ldcg(pmax + b));
    for (int o = 16; o > 0; o >>= 1) fm = fmax(fm, __shfl_down_sync(0xffffffffu, fm, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = fm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x) / 32; ++w) mx = fmax(mx, wmax[w]);
        const double fv = sums[0] / nrep, fd = sums[1] / nrep;
        scal[0] = fv;
        scal[1] = fd;
        scal[2] = mx;
        scal[3] = fv < 0.0 ? 0.0 : fv / fd;
        const long long it = ctl->iters + 1;
        ctl->iters = it;
        if (mx < ftol || it >= itrmax) ctl->done = 1;
        *cnt = 0u;
    }
}

// Unless stopped: the spins of the next iteration into mn, the interior images
// moved with v = lam F (lam = scal[3]) and F the force of the iteration, r = m +
// F (lam dt + dt^2 / (2 mass)) normalised; the end images copied.
__global__ void __launch_bounds__(256) k_gneb_move(const double* __restrict__ m, double* __restrict__ mn,
                                                   const double* __restrict__ F, const double* __restrict__ scal,
                                                   const GnebCtl* ctl, GnebIdx X, int nrep, double dt, double mass) {
    if (ctl->done) return;
    const int r = blockIdx.y;
    const int64_t li = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (li >= X.n) return;
    const int64_t i = r * X.is + li;
    const double3 m0 = ld3(m, i, X.cs);
    if (r == 0 || r == nrep - 1) {
        st3(mn, i, X.cs, m0);
        return;
    }
    const double3 f = ld3(F, i, X.cs);
    const double c = scal[3] * dt + 0.5 / mass * dt * dt;
    double3 v = make_double3(m0.x + f.x * c, m0.y + f.y * c, m0.z + f.z * c);
    const double nr = sqrt(dot(v, v));
    if (nr > 1e-30) v = make_double3(v.x / nr, v.y / nr, v.z / nr);
    st3(mn, i, X.cs, v);
}

// The relaxation of the path in m (nrep images, X) by find_path; the field of
// the images comes from fl (see the header).  The path is left in m.  chunk:
// iterations per graph replay (even).
template <class Fields>
mj_status gneb_relax(Fields& fl, double* m, int nrep, GnebIdx X, int num_sms, cudaStream_t s, const mj_gneb_params* p,
                     int chunk, double* rx, double* ene, double* dene, int64_t* iterations, double* max_force,
                     int32_t* climbing) {
    const double spring = p->spring, dt = p->dt, mass = p->mass, ftol = p->ftol;
    const int64_t itrmax = p->itrmax;
    const int32_t en_zero = p->en_zero;
    const int climb = p->climb ? 1 : 0;
    const int64_t n = X.n, Ntot = n * nrep;  // elements per component over all images
    const int nblk = static_cast<int>((n + 255) / 256);
    const int nbv = nblk * nrep;
    const int n3b = static_cast<int>((3 * Ntot + 255) / 256);
    // F1 / F2 the forces and m / mB the spins of alternate iterations, tau the
    // tangents of the forces before the first move and of the outputs (3 Ntot
    // each, the layout of m); E, pl, fp per image, img the iteration's six path
    // sums per image, scal (v.F, F.F, max |F|, lam); part / part2 block
    // partials; cnt the last-block counters; ctl the stop flag
    double *F1 = nullptr, *F2 = nullptr, *mB = nullptr, *tau = nullptr, *E = nullptr, *part = nullptr,
           *part2 = nullptr;
    unsigned int* cnt = nullptr;
    GnebCtl* ctl = nullptr;
    GnebCtl* hctl = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaGraphExec_t exec = nullptr;
    mj_status st = MJ_OK;
    double** bufs[] = {&F1, &F2, &mB, &tau};
    for (double** q : bufs)
        if (st == MJ_OK) st = cuda_status(cudaMalloc(q, sizeof(double) * 3 * Ntot), "GNEB buffers");
    if (st == MJ_OK) st = cuda_status(cudaMalloc(&E, sizeof(double) * (9 * nrep + 4)), "GNEB buffers");
    if (st == MJ_OK) st = cuda_status(cudaMalloc(&part, sizeof(double) * 6 * nbv), "GNEB buffers");
    if (st == MJ_OK) st = cuda_status(cudaMalloc(&part2, sizeof(double) * std::max(3 * nbv, n3b)), "GNEB buffers");
    if (st == MJ_OK) st = cuda_status(cudaMalloc(&cnt, sizeof(unsigned int) * (nrep + 1)), "GNEB buffers");
    if (st == MJ_OK) st = cuda_status(cudaMalloc(&ctl, sizeof(GnebCtl)), "GNEB buffers");
    if (st == MJ_OK) st = cuda_status(cudaMallocHost(&hctl, 2 * sizeof(GnebCtl)), "GNEB buffers");
    for (int q = 0; q < 2 && st == MJ_OK; ++q)
        st = cuda_status(cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming), "GNEB events");
    auto release = [&]() {
        if (exec) cudaGraphExecDestroy(exec);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        cudaFreeHost(hctl);
        for (double* b : {F1, F2, mB, tau, E, part, part2}) cudaFree(b);
        cudaFree(cnt);
        cudaFree(ctl);
    };
    if (st != MJ_OK) {
        release();
        return st;
    }
    double* pl = E + nrep;
    double* fp = E + 2 * nrep;
    double* img = E + 3 * nrep;
    double* scal = E + 9 * nrep;
    GnebCtl c0;
    std::memset(&c0, 0, sizeof(c0));
    cudaMemsetAsync(scal, 0, sizeof(double) * 4, s);
    cudaMemsetAsync(cnt, 0, sizeof(unsigned int) * (nrep + 1), s);
    cudaMemcpyAsync(ctl, &c0, sizeof(c0), cudaMemcpyHostToDevice, s);
    const dim3 gi(nblk, nrep), gs(nblk, nrep - 1);
    // field, path length pl, tangents of the given mode, fp = F.tau per image
    auto forces = [&](double* F, int mode) -> mj_status {
        mj_status e = fl.field(F, m, E);
        if (e != MJ_OK) return e;
        k_gneb_seg<<<gs, 256, 0, s>>>(m, X, part);
        k_gneb_pathlen<<<1, 256, 0, s>>>(part, nblk, nrep, pl);
        k_gneb_tau<<<gi, 256, 0, s>>>(m, X, nrep, E, mode, tau, part2);
        k_gneb_norm_sum<<<nrep, 256, 0, s>>>(part2, nblk);
        k_gneb_scale<<<gi, 256, 0, s>>>(tau, X, part2, nblk);
        k_gneb_dot<<<gi, 256, 0, s>>>(F, tau, X, part);
        k_gneb_dot_img<<<nrep, 256, 0, s>>>(part, nblk, fp);
        return cuda_status(cudaGetLastError(), "GNEB forces");
    };
    // initial forces: every image's projected field, the GNEB force of the interior
    // ones; max |F| over them all (the convergence check before any move)
    if ((st = forces(F1, 0)) != MJ_OK) {
        release();
        return st;
    }
    k_gneb_force<<<gi, 256, 0, s>>>(F1, tau, fp, pl, E, X, nrep, spring, 1, climb);
    k_gneb_absmax<<<n3b, 256, 0, s>>>(F1, 3 * Ntot, part2);
    k_gneb_maxof<<<1, 256, 0, s>>>(part2, n3b, scal + 2);
    double h0[4];
    cudaMemcpyAsync(h0, E, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h0 + 1, E + nrep - 1, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h0 + 2, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s);
    if ((st = cuda_status(cudaStreamSynchronize(s), "GNEB initial forces")) != MJ_OK) {
        release();
        return st;
    }
    const double E_first = h0[0], E_last = h0[1];
    double fchk = h0[2];
    int64_t done = 0;
    if (itrmax > 0) {
        // the first move (lam = 0: the velocity starts at zero) into mB, then
        // chunks of iterations replayed as one graph: the field with the path
        // sums, k_gneb_step, k_gneb_move.  Forces and spins alternate between
        // their two buffers (an even chunk starts each replay on F1 and mB).  Two
        // chunks are in flight: the stop flag of one is read while the next
        // runs; the iterations after the stop do no work but the field.
        // Four sites per thread once that still gives two blocks per SM: the
        // loads of four sites in flight before each block's reduction.
        const bool spt4 = Ntot >= 2LL * 1024 * num_sms;
        const dim3 gt(nrep, static_cast<unsigned>(spt4 ? (n + 1023) / 1024 : nblk));
        k_gneb_move<<<gi, 256, 0, s>>>(m, mB, F1, scal, ctl, X, nrep, dt, mass);
        st = cuda_status(cudaGetLastError(), "k_gneb_move");
        if (st == MJ_OK) st = cuda_status(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        if (st == MJ_OK) {
            mj_status inner = MJ_OK;
            for (int k = 0; k < chunk && inner == MJ_OK; ++k) {
                double* Fo = (k & 1) ? F2 : F1;
                double* Fn = (k & 1) ? F1 : F2;
                double* mc = (k & 1) ? m : mB;
                double* mo = (k & 1) ? mB : m;
                inner = fl.iterate(Fn, mc, E, img, ctl);
                if (inner != MJ_OK) break;
                const long long im = static_cast<long long>(itrmax);
                if (spt4)
                    k_gneb_step<4><<<gt, 256, 0, s>>>(mc, mo, Fo, Fn, E, img, X, nrep, spring, dt, mass, ftol, im, climb,
                                                      part2, part2 + 2 * nbv, cnt + nrep, ctl, scal);
                else
                    k_gneb_step<1><<<gt, 256, 0, s>>>(mc, mo, Fo, Fn, E, img, X, nrep, spring, dt, mass, ftol, im, climb,
                                                      part2, part2 + 2 * nbv, cnt + nrep, ctl, scal);
                k_gneb_move<<<gi, 256, 0, s>>>(mc, mo, Fn, scal, ctl, X, nrep, dt, mass);
                inner = cuda_status(cudaGetLastError(), "GNEB iteration");
            }
            cudaGraph_t graph = nullptr;
            const cudaError_t e = cudaStreamEndCapture(s, &graph);
            if (inner != MJ_OK) st = inner;
            else if ((st = cuda_status(e, "end capture")) == MJ_OK)
                st = cuda_status(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
            if (graph) cudaGraphDestroy(graph);
        }
        // chunk q: replay, its flag into hctl[q & 1], event ev[q & 1]
        auto launch = [&](int64_t q) -> mj_status {
            mj_status e = cuda_status(cudaGraphLaunch(exec, s), "GNEB graph launch");
            if (e != MJ_OK) return e;
            cudaMemcpyAsync(hctl + (q & 1), ctl, sizeof(GnebCtl), cudaMemcpyDeviceToHost, s);
            return cuda_status(cudaEventRecord(ev[q & 1], s), "GNEB event");
        };
        if (st == MJ_OK) st = launch(0);
        if (st == MJ_OK) st = launch(1);
        for (int64_t q = 0; st == MJ_OK; ++q) {
            if ((st = cuda_status(cudaEventSynchronize(ev[q & 1]), "GNEB iterations")) != MJ_OK) break;
            const GnebCtl hc = hctl[q & 1];
            done = hc.iters;
            if (hc.done) break;
            if (hc.iters != (q + 1) * chunk) {
                st = set_error(MJ_ERR_CUDA, "GNEB iterations did not advance");
                break;
            }
            st = launch(q + 2);
        }
        // the chunk still in flight (or, after an error, all queued work) ends first
        const mj_status fin = cuda_status(cudaStreamSynchronize(s), "GNEB iterations");
        if (st == MJ_OK) st = fin;
        // the relaxed path is in mB after an odd number of iterations
        if (st == MJ_OK && (done & 1))
            cudaMemcpyAsync(m, mB, sizeof(double) * 3 * Ntot, cudaMemcpyDeviceToDevice, s);
        if (st == MJ_OK) {
            cudaMemcpyAsync(&fchk, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s);
            st = cuda_status(cudaStreamSynchronize(s), "GNEB force");
        }
    }
    // outputs (en_path.out): path length, energy above the reference image, and the
    // derivative along the path -F.tau of the final images' projected fields along
    // the simple tangent (lattice_single); the end images' forces are zero after a
    // move, their projected fields before any
    std::vector<double> h(3 * nrep);
    if (st == MJ_OK) st = forces(F2, 1);
    if (st == MJ_OK) {
        cudaMemcpyAsync(h.data(), E, sizeof(double) * 3 * nrep, cudaMemcpyDeviceToHost, s);
        st = cuda_status(cudaStreamSynchronize(s), "GNEB outputs");
    }
    if (st == MJ_OK) {
        const double eref = en_zero == 'I' ? E_first : (en_zero == 'F' ? E_last : 0.0);
        auto en = [&](int r) { return r == 0 ? E_first : (r == nrep - 1 ? E_last : h[r]); };
        for (int r = 0; r < nrep; ++r) {
            rx[r] = h[nrep + r];
            ene[r] = en(r) - eref;
            dene[r] = (r == 0 || r == nrep - 1) && done > 0 ? 0.0 : -h[2 * nrep + r];
        }
        if (iterations) *iterations = done;
        if (max_force) *max_force = fchk;
        // the climbing image of the last iteration (the image energies it saw)
        if (climbing) {
            int c = 0;
            for (int r = 1; r < nrep; ++r)
                if (en(r) > en(c)) c = r;
            *climbing = climb ? c : -1;
        }
    }
    release();
    return st;
}

// the argument checks of both entry points
inline mj_status gneb_check(const mj_gneb_params* p, int nrep, const double* rx, const double* ene,
                            const double* dene) {
    if (!p || !rx || !ene || !dene || nrep < 3 || !(p->dt > 0.0) || !(p->mass > 0.0) || p->itrmax < 0 ||
        (p->en_zero != 'I' && p->en_zero != 'F' && p->en_zero != 'N'))
        return set_error(MJ_ERR_ARG, "bad GNEB arguments (3 or more images, dt > 0, mass > 0, en_zero I/F/N)");
    return MJ_OK;
}

}  // namespace
}  // namespace mj
