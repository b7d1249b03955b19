// Dipolar field as a zero-padded FFT convolution (one magnetic atom per cell).
//
// Reference route (paths relative to Matjes src/): the K tensor of
// Energy/dipolar_magnetic.f90:58-177 on the N_rep grid of
// Hamiltonian_type/fft_ham_base.f90:191-220 (open axes doubled, periodic axes
// with images), K_F = FFT(K)/prod(N_rep) once (fft_ham_fftw.f90:134-178,
// cuda_fft.cpp:96-143), and per call pad -> D2Z -> H_F = K_F M_F -> Z2D ->
// unpack (fft_ham_fftw.f90:239-262, cuda_fft.cu:38-70, fft_ham_internal.f90).
//
// Here the 3D transform of the padded spins is split by axis so that the zero
// planes of an open z axis cost nothing: 2D real transforms over (y, x) of the
// Lz lattice planes only, then complex transforms of length N_rep,z along z
// (the planes z >= Lz of that buffer are zero once and never written).  The
// inverse runs the z transforms and then 2D inverse transforms of the Lz
// planes the consumers read.  Layouts are z-major, [z][component][y][x], so
// that one batched plan covers every (plane, component).  When K is even on
// the N_rep grid (K(-r) = K(r), e.g. open axes without images) K_F is real and
// the pointwise product reads 6 real instead of 6 complex values per wave
// vector; with periodic axes the reference's truncated image sums leave K
// slightly uneven (imaginary parts of K_F ~1e-7 of its scale), and the complex
// product is kept whenever they exceed 1e-13.  The unpack is fused into the consumers: the field and
// step kernels read H on the padded (y, x) grid of the lattice planes.
//
// When N_rep,z is a power of two up to 32 the z transforms and the pointwise
// product are one kernel (k_zconv): one warp per (ky, kx) column, lane = z,
// a radix-2 FFT across the lanes by shuffles (forward in decimation in
// frequency, which leaves the spectrum in bit-reversed order, K_F stored per
// column in that order, inverse in decimation in time back to natural order).
// It reads only the Lz lattice planes of the 2D spectra (the others are the
// zero padding) and writes only the Lz planes the inverse 2D transform reads.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "mj_internal.hpp"

namespace mj {
namespace {

struct DipolarPlan {
    int nrep[3];        // padded grid (x, y, z)
    int lz = 1;         // lattice planes
    int64_t pr = 0;     // real plane: nrep_y * nrep_x
    int64_t pc = 0;     // complex plane: nrep_y * (nrep_x/2 + 1)
    bool real_kf = true;
    double* d_pad = nullptr;               // [lz][3][y][x] real, zero outside the lattice
    double* d_h = nullptr;                 // [lz][3][y][x] real, H of the lattice planes
    cufftDoubleComplex* d_cx = nullptr;    // [nrz][3][y][kx]: 2D spectra, planes >= lz stay zero
    cufftDoubleComplex* d_cz = nullptr;    // [nrz][3][y][kx]: full spectrum, then H's z transform
    double* d_kfr = nullptr;               // [6][nrz][y][kx] real K_F (xx xy xz yy yz zz)
    cufftDoubleComplex* d_kfc = nullptr;   // complex K_F when it is not real
    cufftHandle f2d = 0, fz = 0, b2d = 0;
    bool have_f2d = false, have_fz = false, have_b2d = false;
    // the fused z convolution: K_F per column [pc][nz][6] (kz in bit-reversed
    // order), real or complex, and the twiddles exp(-2 pi i m / nz), m < nz / 2
    bool zconv = false;
    double* d_kzr = nullptr;
    cufftDoubleComplex* d_kzc = nullptr;
    double tw[32] = {};
};

__global__ void k_pad(const double* __restrict__ m, double* __restrict__ pad, int Lx, int Ly, int Lz, int px,
                      int64_t pr) {
    const int64_t N = static_cast<int64_t>(Lx) * Ly * Lz;
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= N) return;
    const int x = static_cast<int>(i % Lx);
    const int64_t r = i / Lx;
    const int y = static_cast<int>(r % Ly);
    const int z = static_cast<int>(r / Ly);
    const int64_t q = x + static_cast<int64_t>(px) * y + 3 * pr * z;
    pad[q] = __ldg(m + i);
    pad[pr + q] = __ldg(m + N + i);
    pad[2 * pr + q] = __ldg(m + 2 * N + i);
}

__device__ __forceinline__ cufftDoubleComplex cmul(cufftDoubleComplex a, cufftDoubleComplex b) {
    return make_cuDoubleComplex(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ cufftDoubleComplex cfma(cufftDoubleComplex a, cufftDoubleComplex b, cufftDoubleComplex c) {
    return make_cuDoubleComplex(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ cufftDoubleComplex rfma(double a, cufftDoubleComplex b, cufftDoubleComplex c) {
    return make_cuDoubleComplex(fma(a, b.x, c.x), fma(a, b.y, c.y));
}

// H_F = K_F M_F over the spectrum [kz][c][ky][kx] (in place), K_F real [6][kz][ky][kx]
__global__ void k_pointwise_real(cufftDoubleComplex* __restrict__ spec, const double* __restrict__ kf, int64_t pc,
                                 int64_t nkc) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= nkc) return;
    const int64_t kz = k / pc, w = k - kz * pc;
    cufftDoubleComplex* s = spec + kz * 3 * pc + w;
    const cufftDoubleComplex mx = s[0], my = s[pc], mz = s[2 * pc];
    const double kxx = __ldg(kf + k), kxy = __ldg(kf + nkc + k), kxz = __ldg(kf + 2 * nkc + k);
    const double kyy = __ldg(kf + 3 * nkc + k), kyz = __ldg(kf + 4 * nkc + k), kzz = __ldg(kf + 5 * nkc + k);
    const cufftDoubleComplex z0 = make_cuDoubleComplex(0.0, 0.0);
    s[0] = rfma(kxx, mx, rfma(kxy, my, rfma(kxz, mz, z0)));
    s[pc] = rfma(kxy, mx, rfma(kyy, my, rfma(kyz, mz, z0)));
    s[2 * pc] = rfma(kxz, mx, rfma(kyz, my, rfma(kzz, mz, z0)));
}

__global__ void k_pointwise_cplx(cufftDoubleComplex* __restrict__ spec, const cufftDoubleComplex* __restrict__ kf,
                                 int64_t pc, int64_t nkc) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= nkc) return;
    const int64_t kz = k / pc, w = k - kz * pc;
    cufftDoubleComplex* s = spec + kz * 3 * pc + w;
    const cufftDoubleComplex mx = s[0], my = s[pc], mz = s[2 * pc];
    const cufftDoubleComplex kxx = kf[k], kxy = kf[nkc + k], kxz = kf[2 * nkc + k];
    const cufftDoubleComplex kyy = kf[3 * nkc + k], kyz = kf[4 * nkc + k], kzz = kf[5 * nkc + k];
    s[0] = cfma(kxx, mx, cfma(kxy, my, cmul(kxz, mz)));
    s[pc] = cfma(kxy, mx, cfma(kyy, my, cmul(kyz, mz)));
    s[2 * pc] = cfma(kxz, mx, cfma(kyz, my, cmul(kzz, mz)));
}

__global__ void k_scale(cufftDoubleComplex* __restrict__ a, int64_t n, double s) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    a[k].x *= s;
    a[k].y *= s;
}

// Twiddles of a length-NZ transform: (cos, sin) of -2 pi m / NZ, m < NZ/2
struct ZTwiddle {
    double c[16], s[16];
};

__device__ __forceinline__ double2 shfl_xor_c(double2 v, int h) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, h), __shfl_xor_sync(0xffffffffu, v.y, h));
}
__device__ __forceinline__ double2 cmul_d(double2 a, double c, double s) {  // a (c + i s)
    return make_double2(fma(a.x, c, -(a.y * s)), fma(a.x, s, a.y * c));
}

// The forward transform of the lanes' values (lane l of a group of NZ holds
// element l): decimation in frequency, lane l ends with X(bitrev(l)).
template <int NZ>
__device__ __forceinline__ double2 zfft_forward(double2 x, int l, const double2* __restrict__ tw) {
#pragma unroll
    for (int h = NZ / 2; h >= 1; h >>= 1) {
        const double2 p = shfl_xor_c(x, h);
        if (l & h) {
            const double2 w = tw[(l & (h - 1)) * (NZ / (2 * h))];
            x = cmul_d(make_double2(p.x - x.x, p.y - x.y), w.x, w.y);
        } else {
            x = make_double2(x.x + p.x, x.y + p.y);
        }
    }
    return x;
}

// The inverse (exp(+2 pi i ...), unscaled) of bit-reversed lanes: decimation
// in time, lane l ends with y(l).
template <int NZ>
__device__ __forceinline__ double2 zfft_inverse(double2 x, int l, const double2* __restrict__ tw) {
#pragma unroll
    for (int h = 1; h < NZ; h <<= 1) {
        const double2 w = tw[(l & (h - 1)) * (NZ / (2 * h))];
        const double2 t = (l & h) ? cmul_d(x, w.x, -w.y) : x;
        const double2 p = shfl_xor_c(t, h);
        x = (l & h) ? make_double2(p.x - t.x, p.y - t.y) : make_double2(t.x + p.x, t.y + p.y);
    }
    return x;
}

// z transforms and the product H_F = K_F M_F in one pass: spec_in [z][c][col]
// (planes z < lz), out [z][c][col] (planes z < lz), K_F [col][6][l] with l the
// lane (bit-reversed kz); REAL: K_F real.  A block of 8 warps takes C = 256/NZ
// consecutive columns, one column per NZ lanes (every lane one z): the rows
// (z, c) of its columns are read and written whole through shared memory,
// [z][c * C + column] with rows of 3 C + 1 16-byte slots, so that the lanes of
// one column hit distinct banks.
template <int NZ>
struct ZcGeom {
    static constexpr int C = 256 / NZ;   // columns per block
    static constexpr int ROW = 3 * C + 1;
    static constexpr size_t smem = sizeof(double2) * NZ * ROW;
};

template <int NZ, bool REAL>
__global__ void __launch_bounds__(256) k_zconv(const double2* __restrict__ in, double2* __restrict__ out,
                                               const double* __restrict__ kr, const double2* __restrict__ kc,
                                               int64_t pc, int lz, const ZTwiddle W) {
    using Z = ZcGeom<NZ>;
    extern __shared__ double2 zs[];  // [NZ][ROW]
    // the twiddles in shared memory (the lanes index them differently)
    __shared__ double2 tw[16];
    if (threadIdx.x < NZ / 2) tw[threadIdx.x] = make_double2(W.c[threadIdx.x], W.s[threadIdx.x]);
    const int64_t col0 = static_cast<int64_t>(blockIdx.x) * Z::C;
    const int ncol = pc - col0 < Z::C ? static_cast<int>(pc - col0) : Z::C;
    // rows (z, c), z < lz: consecutive threads on consecutive columns of a row
    for (int idx = threadIdx.x; idx < 3 * lz * Z::C; idx += blockDim.x) {
        const int row = idx / Z::C, q = idx - row * Z::C;
        const int z = row / 3, c = row - 3 * z;
        zs[z * Z::ROW + c * Z::C + q] =
            q < ncol ? in[(static_cast<int64_t>(z) * 3 + c) * pc + col0 + q] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const int l = threadIdx.x % NZ, q = threadIdx.x / NZ;  // this lane's z and column
    const int64_t col = col0 + (q < ncol ? q : 0);
    double2 v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        v[c] = l < lz ? zs[l * Z::ROW + c * Z::C + q] : make_double2(0.0, 0.0);
        v[c] = zfft_forward<NZ>(v[c], l, tw);
    }
    double2 h[3];
    if constexpr (REAL) {
        const double* k = kr + col * 6 * NZ + l;
        const double kxx = __ldg(k), kxy = __ldg(k + NZ), kxz = __ldg(k + 2 * NZ), kyy = __ldg(k + 3 * NZ),
                     kyz = __ldg(k + 4 * NZ), kzz = __ldg(k + 5 * NZ);
        h[0] = make_double2(fma(kxx, v[0].x, fma(kxy, v[1].x, kxz * v[2].x)),
                            fma(kxx, v[0].y, fma(kxy, v[1].y, kxz * v[2].y)));
        h[1] = make_double2(fma(kxy, v[0].x, fma(kyy, v[1].x, kyz * v[2].x)),
                            fma(kxy, v[0].y, fma(kyy, v[1].y, kyz * v[2].y)));
        h[2] = make_double2(fma(kxz, v[0].x, fma(kyz, v[1].x, kzz * v[2].x)),
                            fma(kxz, v[0].y, fma(kyz, v[1].y, kzz * v[2].y)));
    } else {
        const double2* k = kc + col * 6 * NZ + l;
        const double2 kxx = k[0], kxy = k[NZ], kxz = k[2 * NZ], kyy = k[3 * NZ], kyz = k[4 * NZ], kzz = k[5 * NZ];
        auto mac = [](double2 a, double2 b, double2 acc) {
            return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
        };
        const double2 z0 = make_double2(0.0, 0.0);
        h[0] = mac(kxx, v[0], mac(kxy, v[1], mac(kxz, v[2], z0)));
        h[1] = mac(kxy, v[0], mac(kyy, v[1], mac(kyz, v[2], z0)));
        h[2] = mac(kxz, v[0], mac(kyz, v[1], mac(kzz, v[2], z0)));
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double2 y = zfft_inverse<NZ>(h[c], l, tw);
        if (l < lz) zs[l * Z::ROW + c * Z::C + q] = y;  // this lane's own slot, read above by it alone
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < 3 * lz * Z::C; idx += blockDim.x) {
        const int row = idx / Z::C, q2 = idx - row * Z::C;
        const int z = row / 3, c = row - 3 * z;
        if (q2 < ncol) out[(static_cast<int64_t>(z) * 3 + c) * pc + col0 + q2] = zs[z * Z::ROW + c * Z::C + q2];
    }
}

mj_status cufft_status(cufftResult r, const char* where) {
    if (r == CUFFT_SUCCESS) return MJ_OK;
    return set_error(MJ_ERR_CUDA, std::string("cuFFT error ") + std::to_string(static_cast<int>(r)) + " in " + where);
}

void free_plan(DipolarPlan* d) {
    if (!d) return;
    if (d->have_f2d) cufftDestroy(d->f2d);
    if (d->have_fz) cufftDestroy(d->fz);
    if (d->have_b2d) cufftDestroy(d->b2d);
    cudaFree(d->d_pad);
    cudaFree(d->d_h);
    cudaFree(d->d_cx);
    cudaFree(d->d_cz);
    cudaFree(d->d_kfr);
    cudaFree(d->d_kfc);
    cudaFree(d->d_kzr);
    cudaFree(d->d_kzc);
    delete d;
}

}  // namespace

mj_status dipolar_create(mj_plan* p, const std::vector<double>& K, cudaStream_t s) {
    DipolarPlan* d = new DipolarPlan();
    for (int k = 0; k < 3; ++k) d->nrep[k] = p->nrep[k];
    d->lz = p->sp.L[2];
    const int nx = d->nrep[0], ny = d->nrep[1], nz = d->nrep[2];
    const int nkx = nx / 2 + 1;
    d->pr = static_cast<int64_t>(ny) * nx;
    d->pc = static_cast<int64_t>(ny) * nkx;
    const int64_t nk = d->pr * nz, nkc = d->pc * nz;
    mj_status st = MJ_OK;
    auto fail = [&](mj_status e) {
        free_plan(d);
        return e;
    };
    if (d->lz > nz) return fail(set_error(MJ_ERR_ARG, "dipolar grid smaller than the lattice"));
    auto al = [&](auto** ptr, size_t bytes, const char* what) {
        return cuda_status(cudaMalloc(reinterpret_cast<void**>(ptr), bytes), what);
    };
    if ((st = al(&d->d_pad, sizeof(double) * 3 * d->pr * d->lz, "dipolar pad")) != MJ_OK ||
        (st = al(&d->d_h, sizeof(double) * 3 * d->pr * d->lz, "dipolar H")) != MJ_OK ||
        (st = al(&d->d_cx, sizeof(cufftDoubleComplex) * 3 * nkc, "dipolar spectra")) != MJ_OK ||
        (st = al(&d->d_cz, sizeof(cufftDoubleComplex) * 3 * nkc, "dipolar spectra")) != MJ_OK)
        return fail(st);
    // zero once: the pad outside the lattice rows/columns and the spectra planes z >= Lz
    if ((st = cuda_status(cudaMemsetAsync(d->d_pad, 0, sizeof(double) * 3 * d->pr * d->lz, s), "dipolar memset")) != MJ_OK ||
        (st = cuda_status(cudaMemsetAsync(d->d_cx, 0, sizeof(cufftDoubleComplex) * 3 * nkc, s), "dipolar memset")) != MJ_OK)
        return fail(st);

    // K_F of the six unique components on the full grid (3D transform, once), scaled by 1/prod(N_rep)
    cufftDoubleComplex* kf = nullptr;
    {
        std::vector<double> k6(static_cast<size_t>(6) * nk);
        const int sel[6] = {0, 1, 2, 4, 5, 8};
        for (int c = 0; c < 6; ++c)
            for (int64_t q = 0; q < nk; ++q) k6[static_cast<size_t>(c) * nk + q] = K[static_cast<size_t>(q) * 9 + sel[c]];
        double* d_k6 = nullptr;
        if ((st = al(&d_k6, sizeof(double) * 6 * nk, "dipolar K")) != MJ_OK) return fail(st);
        if ((st = al(&kf, sizeof(cufftDoubleComplex) * 6 * nkc, "dipolar K_F")) != MJ_OK) {
            cudaFree(d_k6);
            return fail(st);
        }
        int dims[3] = {nz, ny, nx}, inembed[3] = {nz, ny, nx}, onembed[3] = {nz, ny, nkx};
        cufftHandle pk;
        cufftResult r = cudaMemcpyAsync(d_k6, k6.data(), sizeof(double) * 6 * nk, cudaMemcpyHostToDevice, s) == cudaSuccess
                            ? cufftPlanMany(&pk, 3, dims, inembed, 1, static_cast<int>(nk), onembed, 1,
                                            static_cast<int>(nkc), CUFFT_D2Z, 6)
                            : CUFFT_EXEC_FAILED;
        if (r == CUFFT_SUCCESS) {
            cufftSetStream(pk, s);
            r = cufftExecD2Z(pk, d_k6, kf);
            if (r == CUFFT_SUCCESS)
                k_scale<<<static_cast<unsigned>((6 * nkc + 255) / 256), 256, 0, s>>>(kf, 6 * nkc, 1.0 / static_cast<double>(nk));
            cudaStreamSynchronize(s);
            cufftDestroy(pk);
        }
        cudaFree(d_k6);
        if (r != CUFFT_SUCCESS) {
            cudaFree(kf);
            return fail(cufft_status(r, "K transform"));
        }
    }
    // real when the imaginary parts are rounding: keep 6 real values per wave vector
    {
        std::vector<cufftDoubleComplex> h(static_cast<size_t>(6) * nkc);
        if ((st = cuda_status(cudaMemcpy(h.data(), kf, sizeof(cufftDoubleComplex) * h.size(), cudaMemcpyDeviceToHost),
                              "K_F download")) != MJ_OK) {
            cudaFree(kf);
            return fail(st);
        }
        double re = 0.0, im = 0.0;
        for (const cufftDoubleComplex& c : h) {
            re = std::max(re, std::fabs(c.x));
            im = std::max(im, std::fabs(c.y));
        }
        d->real_kf = im <= 1e-13 * re;
        // the fused z convolution's K_F: per column, kz in the lanes' bit-reversed order
        if (nz >= 2 && nz <= 32 && (nz & (nz - 1)) == 0) {
            int bits = 0;
            while ((1 << bits) < nz) ++bits;
            auto bitrev = [&](int l) {
                int r = 0;
                for (int b = 0; b < bits; ++b) r |= ((l >> b) & 1) << (bits - 1 - b);
                return r;
            };
            const size_t ncol = static_cast<size_t>(d->pc);
            if (d->real_kf) {
                std::vector<double> kz(ncol * nz * 6);
                for (size_t col = 0; col < ncol; ++col)
                    for (int c = 0; c < 6; ++c)
                        for (int l = 0; l < nz; ++l)
                            kz[(col * 6 + c) * nz + l] =
                                h[static_cast<size_t>(c) * nkc + static_cast<size_t>(bitrev(l)) * ncol + col].x;
                st = al(&d->d_kzr, sizeof(double) * kz.size(), "dipolar K_F columns");
                if (st == MJ_OK)
                    st = cuda_status(cudaMemcpy(d->d_kzr, kz.data(), sizeof(double) * kz.size(), cudaMemcpyHostToDevice),
                                     "K_F columns upload");
            } else {
                std::vector<cufftDoubleComplex> kz(ncol * nz * 6);
                for (size_t col = 0; col < ncol; ++col)
                    for (int c = 0; c < 6; ++c)
                        for (int l = 0; l < nz; ++l)
                            kz[(col * 6 + c) * nz + l] =
                                h[static_cast<size_t>(c) * nkc + static_cast<size_t>(bitrev(l)) * ncol + col];
                st = al(&d->d_kzc, sizeof(cufftDoubleComplex) * kz.size(), "dipolar K_F columns");
                if (st == MJ_OK)
                    st = cuda_status(cudaMemcpy(d->d_kzc, kz.data(), sizeof(cufftDoubleComplex) * kz.size(),
                                                cudaMemcpyHostToDevice),
                                     "K_F columns upload");
            }
            if (st != MJ_OK) {
                cudaFree(kf);
                return fail(st);
            }
            // exp(-2 pi i m / nz), m < nz / 2, rounded once from long double
            const long double pi = 3.141592653589793238462643383279502884L;
            for (int m = 0; m < nz / 2; ++m) {
                const long double a = 2.0L * pi * static_cast<long double>(m) / static_cast<long double>(nz);
                d->tw[m] = static_cast<double>(std::cos(a));
                d->tw[16 + m] = static_cast<double>(-std::sin(a));
            }
            d->zconv = true;
        }
        if (d->real_kf) {
            std::vector<double> r(h.size());
            for (size_t q = 0; q < h.size(); ++q) r[q] = h[q].x;
            if ((st = al(&d->d_kfr, sizeof(double) * r.size(), "dipolar K_F")) != MJ_OK ||
                (st = cuda_status(cudaMemcpy(d->d_kfr, r.data(), sizeof(double) * r.size(), cudaMemcpyHostToDevice),
                                  "K_F upload")) != MJ_OK) {
                cudaFree(kf);
                return fail(st);
            }
            cudaFree(kf);
        } else {
            d->d_kfc = kf;
        }
    }
    // 2D real transforms over (y, x) of the lattice planes, batched over (z < Lz, component)
    {
        int n2[2] = {ny, nx}, in2[2] = {ny, nx}, on2[2] = {ny, nkx};
        cufftResult r = cufftPlanMany(&d->f2d, 2, n2, in2, 1, static_cast<int>(d->pr), on2, 1, static_cast<int>(d->pc),
                                      CUFFT_D2Z, 3 * d->lz);
        if (r != CUFFT_SUCCESS) return fail(cufft_status(r, "2D forward plan"));
        d->have_f2d = true;
        r = cufftPlanMany(&d->b2d, 2, n2, on2, 1, static_cast<int>(d->pc), in2, 1, static_cast<int>(d->pr), CUFFT_Z2D,
                          3 * d->lz);
        if (r != CUFFT_SUCCESS) return fail(cufft_status(r, "2D backward plan"));
        d->have_b2d = true;
    }
    // complex transforms along z: one line per (component, ky, kx), stride 3 pc
    if (nz > 1) {
        int nz1[1] = {nz}, emb[1] = {nz};
        const int stride = static_cast<int>(3 * d->pc);
        cufftResult r = cufftPlanMany(&d->fz, 1, nz1, emb, stride, 1, emb, stride, 1, CUFFT_Z2Z, stride);
        if (r != CUFFT_SUCCESS) return fail(cufft_status(r, "z plan"));
        d->have_fz = true;
    }
    p->dip = d;
    return MJ_OK;
}

void dipolar_destroy(mj_plan* p) {
    free_plan(static_cast<DipolarPlan*>(p->dip));
    p->dip = nullptr;
}

mj_status dipolar_apply(mj_plan* p, const double* m, double* /*H unused: consumers read the padded grid*/,
                        cudaStream_t s) {
    DipolarPlan* d = static_cast<DipolarPlan*>(p->dip);
    if (!d) return set_error(MJ_ERR_ARG, "dipolar plan missing");
    const int64_t N = p->N;
    const int64_t nkc = d->pc * d->nrep[2];
    mj_status st = MJ_OK;
    // the pass that wrote m may have written the padded grid as well
    if (p->dip_pad_holds != m) {
        k_pad<<<static_cast<unsigned>((N + 255) / 256), 256, 0, s>>>(m, d->d_pad, p->sp.L[0], p->sp.L[1], p->sp.L[2],
                                                                      d->nrep[0], d->pr);
        if ((st = cuda_status(cudaGetLastError(), "k_pad")) != MJ_OK) return st;
    }
    p->dip_pad_holds = nullptr;
    cufftSetStream(d->f2d, s);
    cufftSetStream(d->b2d, s);
    if (d->have_fz) cufftSetStream(d->fz, s);
    // planes z < Lz of d_cx; the rest of it stays zero
    if ((st = cufft_status(cufftExecD2Z(d->f2d, d->d_pad, d->d_cx), "2D D2Z")) != MJ_OK) return st;
    if (d->zconv && p->dip_zconv) {
        // z transforms and product in one pass, into the planes z < Lz of d_cz
        ZTwiddle W;
        for (int m = 0; m < 16; ++m) {
            W.c[m] = d->tw[m];
            W.s[m] = d->tw[16 + m];
        }
        const int nz = d->nrep[2];
        const double2* in = reinterpret_cast<const double2*>(d->d_cx);
        double2* out = reinterpret_cast<double2*>(d->d_cz);
        const double2* kc = reinterpret_cast<const double2*>(d->d_kzc);
        auto go = [&](auto nzc) {
            constexpr int NZ = decltype(nzc)::value;
            using Z = ZcGeom<NZ>;
            const unsigned nb = static_cast<unsigned>((d->pc + Z::C - 1) / Z::C);
            if (d->real_kf) k_zconv<NZ, true><<<nb, 256, Z::smem, s>>>(in, out, d->d_kzr, kc, d->pc, d->lz, W);
            else k_zconv<NZ, false><<<nb, 256, Z::smem, s>>>(in, out, d->d_kzr, kc, d->pc, d->lz, W);
        };
        switch (nz) {
            case 2: go(std::integral_constant<int, 2>{}); break;
            case 4: go(std::integral_constant<int, 4>{}); break;
            case 8: go(std::integral_constant<int, 8>{}); break;
            case 16: go(std::integral_constant<int, 16>{}); break;
            default: go(std::integral_constant<int, 32>{}); break;
        }
        if ((st = cuda_status(cudaGetLastError(), "k_zconv")) != MJ_OK) return st;
        return cufft_status(cufftExecZ2D(d->b2d, d->d_cz, d->d_h), "2D Z2D");
    }
    cufftDoubleComplex* spec = d->d_cx;
    if (d->have_fz) {
        if ((st = cufft_status(cufftExecZ2Z(d->fz, d->d_cx, d->d_cz, CUFFT_FORWARD), "z forward")) != MJ_OK) return st;
        spec = d->d_cz;
    }
    if (d->real_kf)
        k_pointwise_real<<<static_cast<unsigned>((nkc + 255) / 256), 256, 0, s>>>(spec, d->d_kfr, d->pc, nkc);
    else
        k_pointwise_cplx<<<static_cast<unsigned>((nkc + 255) / 256), 256, 0, s>>>(spec, d->d_kfc, d->pc, nkc);
    if ((st = cuda_status(cudaGetLastError(), "k_pointwise")) != MJ_OK) return st;
    if (d->have_fz && (st = cufft_status(cufftExecZ2Z(d->fz, d->d_cz, d->d_cz, CUFFT_INVERSE), "z inverse")) != MJ_OK)
        return st;
    // H of the lattice planes: the first 3 Lz complex planes of the spectrum
    return cufft_status(cufftExecZ2D(d->b2d, spec, d->d_h), "2D Z2D");
}

DipPad dipolar_pad(const mj_plan* p) {
    const DipolarPlan* d = static_cast<const DipolarPlan*>(p->dip);
    if (!p->dip_on || !d) return DipPad{nullptr, 0, 0, 0};
    return DipPad{d->d_pad, d->pr, 3 * d->pr, d->nrep[0]};
}

DipView dipolar_view(const mj_plan* p) {
    DipView v;
    const DipolarPlan* d = static_cast<const DipolarPlan*>(p->dip);
    if (!p->dip_on || !d) {
        v.h = nullptr;
        v.cs = v.zs = 0;
        v.px = 0;
        return v;
    }
    v.h = d->d_h;
    v.cs = d->pr;
    v.zs = 3 * d->pr;
    v.px = d->nrep[0];
    return v;
}

}  // namespace mj
