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
#include <cufft.h>

#include <algorithm>
#include <cmath>
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
    k_pad<<<static_cast<unsigned>((N + 255) / 256), 256, 0, s>>>(m, d->d_pad, p->sp.L[0], p->sp.L[1], p->sp.L[2],
                                                                  d->nrep[0], d->pr);
    mj_status st = cuda_status(cudaGetLastError(), "k_pad");
    if (st != MJ_OK) return st;
    cufftSetStream(d->f2d, s);
    cufftSetStream(d->b2d, s);
    if (d->have_fz) cufftSetStream(d->fz, s);
    // planes z < Lz of d_cx; the rest of it stays zero
    if ((st = cufft_status(cufftExecD2Z(d->f2d, d->d_pad, d->d_cx), "2D D2Z")) != MJ_OK) return st;
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
