// Dipolar field as a zero-padded FFT convolution (one magnetic atom per cell).
//
// Reference route (paths relative to Matjes src/): the K tensor of
// Energy/dipolar_magnetic.f90:58-177 on the N_rep grid of
// Hamiltonian_type/fft_ham_base.f90:191-220 (open axes doubled, periodic axes
// with images), K_F = FFT(K)/prod(N_rep) once (fft_ham_fftw.f90:134-178,
// cuda_fft.cpp:96-143), and per call pad -> D2Z -> H_F = K_F M_F -> Z2D ->
// unpack (fft_ham_fftw.f90:239-262, cuda_fft.cu:38-70, fft_ham_internal.f90).
//
// Here: cuFFT does the transforms (three components batched in one plan);
// the pad, the pointwise product over the half spectrum with the six unique
// components of the symmetric K_F, and the K_F set-up are hand-written kernels.
// The unpack is fused into the consumers: the field/step kernels read H on the
// padded grid directly.
#include <cufft.h>

#include <vector>

#include "mj_internal.hpp"

namespace mj {
namespace {

struct DipolarPlan {
    int nrep[3];
    int64_t nk = 0, nkc = 0;
    double* d_pad = nullptr;            // [3][nk] real, zero outside the lattice
    double* d_hpad = nullptr;           // [3][nk] real, H on the padded grid
    cufftDoubleComplex* d_spec = nullptr;  // [3][nkc]
    cufftDoubleComplex* d_kf = nullptr;    // [6][nkc]: xx xy xz yy yz zz
    cufftHandle fwd = 0, bwd = 0;
    bool have_fwd = false, have_bwd = false;
};

__global__ void k_pad(const double* __restrict__ m, double* __restrict__ pad, int Lx, int Ly, int Lz, int px, int py,
                      int64_t nk) {
    const int64_t N = static_cast<int64_t>(Lx) * Ly * Lz;
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= N) return;
    const int x = static_cast<int>(i % Lx);
    const int64_t r = i / Lx;
    const int y = static_cast<int>(r % Ly);
    const int z = static_cast<int>(r / Ly);
    const int64_t q = x + static_cast<int64_t>(px) * (y + static_cast<int64_t>(py) * z);
    pad[q] = __ldg(m + i);
    pad[nk + q] = __ldg(m + N + i);
    pad[2 * nk + q] = __ldg(m + 2 * N + i);
}

__device__ __forceinline__ cufftDoubleComplex cmul(cufftDoubleComplex a, cufftDoubleComplex b) {
    return make_cuDoubleComplex(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ cufftDoubleComplex cfma(cufftDoubleComplex a, cufftDoubleComplex b, cufftDoubleComplex c) {
    return make_cuDoubleComplex(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}

// H_F = K_F M_F for the symmetric 3x3 K_F, in place over the spectrum.
__global__ void k_pointwise(cufftDoubleComplex* __restrict__ spec, const cufftDoubleComplex* __restrict__ kf, int64_t nkc) {
    const int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (k >= nkc) return;
    const cufftDoubleComplex mx = spec[k], my = spec[nkc + k], mz = spec[2 * nkc + k];
    const cufftDoubleComplex kxx = kf[k], kxy = kf[nkc + k], kxz = kf[2 * nkc + k];
    const cufftDoubleComplex kyy = kf[3 * nkc + k], kyz = kf[4 * nkc + k], kzz = kf[5 * nkc + k];
    spec[k] = cfma(kxx, mx, cfma(kxy, my, cmul(kxz, mz)));
    spec[nkc + k] = cfma(kxy, mx, cfma(kyy, my, cmul(kyz, mz)));
    spec[2 * nkc + k] = cfma(kxz, mx, cfma(kyz, my, cmul(kzz, mz)));
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
    if (d->have_fwd) cufftDestroy(d->fwd);
    if (d->have_bwd) cufftDestroy(d->bwd);
    cudaFree(d->d_pad);
    cudaFree(d->d_hpad);
    cudaFree(d->d_spec);
    cudaFree(d->d_kf);
    delete d;
}

}  // namespace

mj_status dipolar_create(mj_plan* p, const std::vector<double>& K, cudaStream_t s) {
    DipolarPlan* d = new DipolarPlan();
    for (int k = 0; k < 3; ++k) d->nrep[k] = p->nrep[k];
    d->nk = static_cast<int64_t>(d->nrep[0]) * d->nrep[1] * d->nrep[2];
    d->nkc = static_cast<int64_t>(d->nrep[0] / 2 + 1) * d->nrep[1] * d->nrep[2];
    mj_status st = MJ_OK;
    auto fail = [&](mj_status e) {
        free_plan(d);
        return e;
    };
    if ((st = cuda_status(cudaMalloc(&d->d_pad, sizeof(double) * 3 * d->nk), "dipolar pad")) != MJ_OK) return fail(st);
    if ((st = cuda_status(cudaMalloc(&d->d_hpad, sizeof(double) * 3 * d->nk), "dipolar hpad")) != MJ_OK) return fail(st);
    if ((st = cuda_status(cudaMalloc(&d->d_spec, sizeof(cufftDoubleComplex) * 6 * d->nkc), "dipolar spec")) != MJ_OK)
        return fail(st);
    if ((st = cuda_status(cudaMalloc(&d->d_kf, sizeof(cufftDoubleComplex) * 6 * d->nkc), "dipolar kf")) != MJ_OK)
        return fail(st);
    if ((st = cuda_status(cudaMemsetAsync(d->d_pad, 0, sizeof(double) * 3 * d->nk, s), "dipolar memset")) != MJ_OK)
        return fail(st);
    // cuFFT dims are row-major (slowest first): (z, y, x); x is the fastest lattice axis
    int dims[3] = {d->nrep[2], d->nrep[1], d->nrep[0]};
    int inembed[3] = {d->nrep[2], d->nrep[1], d->nrep[0]};
    int onembed[3] = {d->nrep[2], d->nrep[1], d->nrep[0] / 2 + 1};
    // K: six unique real components -> K_F, normalised by 1/prod(N_rep)
    {
        std::vector<double> k6(static_cast<size_t>(6) * d->nk);
        const int sel[6] = {0, 1, 2, 4, 5, 8};
        for (int c = 0; c < 6; ++c)
            for (int64_t q = 0; q < d->nk; ++q) k6[static_cast<size_t>(c) * d->nk + q] = K[static_cast<size_t>(q) * 9 + sel[c]];
        double* d_k6 = nullptr;
        if ((st = cuda_status(cudaMalloc(&d_k6, sizeof(double) * 6 * d->nk), "dipolar K")) != MJ_OK) return fail(st);
        if ((st = cuda_status(cudaMemcpyAsync(d_k6, k6.data(), sizeof(double) * 6 * d->nk, cudaMemcpyHostToDevice, s),
                              "dipolar K upload")) != MJ_OK) {
            cudaFree(d_k6);
            return fail(st);
        }
        cufftHandle pk;
        cufftResult r = cufftPlanMany(&pk, 3, dims, inembed, 1, static_cast<int>(d->nk), onembed, 1,
                                      static_cast<int>(d->nkc), CUFFT_D2Z, 6);
        if (r != CUFFT_SUCCESS) {
            cudaFree(d_k6);
            return fail(cufft_status(r, "K plan"));
        }
        cufftSetStream(pk, s);
        r = cufftExecD2Z(pk, d_k6, d->d_kf);
        if (r == CUFFT_SUCCESS) {
            const int64_t n = 6 * d->nkc;
            k_scale<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(d->d_kf, n, 1.0 / static_cast<double>(d->nk));
        }
        cudaStreamSynchronize(s);
        cufftDestroy(pk);
        cudaFree(d_k6);
        if (r != CUFFT_SUCCESS) return fail(cufft_status(r, "K transform"));
        if ((st = cuda_status(cudaGetLastError(), "K scale")) != MJ_OK) return fail(st);
    }
    cufftResult r = cufftPlanMany(&d->fwd, 3, dims, inembed, 1, static_cast<int>(d->nk), onembed, 1,
                                  static_cast<int>(d->nkc), CUFFT_D2Z, 3);
    if (r != CUFFT_SUCCESS) return fail(cufft_status(r, "forward plan"));
    d->have_fwd = true;
    r = cufftPlanMany(&d->bwd, 3, dims, onembed, 1, static_cast<int>(d->nkc), inembed, 1, static_cast<int>(d->nk),
                      CUFFT_Z2D, 3);
    if (r != CUFFT_SUCCESS) return fail(cufft_status(r, "backward plan"));
    d->have_bwd = true;
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
    k_pad<<<static_cast<unsigned>((N + 255) / 256), 256, 0, s>>>(m, d->d_pad, p->sp.L[0], p->sp.L[1], p->sp.L[2],
                                                                  d->nrep[0], d->nrep[1], d->nk);
    mj_status st = cuda_status(cudaGetLastError(), "k_pad");
    if (st != MJ_OK) return st;
    cufftSetStream(d->fwd, s);
    cufftSetStream(d->bwd, s);
    if ((st = cufft_status(cufftExecD2Z(d->fwd, d->d_pad, d->d_spec), "D2Z")) != MJ_OK) return st;
    k_pointwise<<<static_cast<unsigned>((d->nkc + 255) / 256), 256, 0, s>>>(d->d_spec, d->d_kf, d->nkc);
    if ((st = cuda_status(cudaGetLastError(), "k_pointwise")) != MJ_OK) return st;
    return cufft_status(cufftExecZ2D(d->bwd, d->d_spec, d->d_hpad), "Z2D");
}

DipView dipolar_view(const mj_plan* p) {
    DipView v;
    const DipolarPlan* d = static_cast<const DipolarPlan*>(p->dip);
    if (!p->dip_on || !d) {
        v.h = nullptr;
        v.nk = 0;
        v.px = v.py = 0;
        return v;
    }
    v.h = d->d_hpad;
    v.nk = d->nk;
    v.px = d->nrep[0];
    v.py = d->nrep[1];
    return v;
}

}  // namespace mj
