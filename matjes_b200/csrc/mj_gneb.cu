// GNEB path relaxation on any plan: find_path of GNEB/gneb_utils.f90:19-240
// with the field of every image from the plan's own field kernels, so the path
// may live on any lattice of one magnetic atom per cell a plan holds (tiled and
// generic stencils, ELL couplings, open boundaries, 3D films) and the images see
// every term of the plan's Hamiltonian, the FFT dipolar term included, as
// get_eff_field and H%energy give them to the reference's GNEB (:77-81,
// :154-157).  The path is nimg images of the plan's N spins in one device
// array, image r the SoA block x[N] | y[N] | z[N] at 3 N r.
//
// Per image one field launch (launch_field: field and total energy); then
// k_gneb_project (before the first move and for the outputs) or k_gneb_sums
// (each iteration: projection and the six path sums per image).  The rest of
// the relaxation is mj_gneb.cuh's, shared with the replica batch.
#include <algorithm>
#include <cstring>

#include "mj_gneb.cuh"
#include "mj_internal.hpp"

namespace mj {
namespace {

struct PlanFields {
    mj_plan* p;
    int nrep;
    GnebIdx X;
    cudaStream_t s;
    double* part;       // path-sum partials: 6 per (image, block)
    unsigned int* cnt;  // last-block counters, one per image

    mj_status images(double* F, const double* m, double* E) {
        for (int r = 0; r < nrep; ++r) {
            const int64_t o = static_cast<int64_t>(r) * X.is;
            mj_status e = launch_field(p, m + o, F + o, nullptr, E + r, s);
            if (e != MJ_OK) return e;
        }
        return MJ_OK;
    }
    mj_status field(double* F, double* m, double* E) {
        mj_status e = images(F, m, E);
        if (e != MJ_OK) return e;
        const int nblk = static_cast<int>((X.n + 255) / 256);
        k_gneb_project<<<dim3(nblk, nrep), 256, 0, s>>>(F, m, X);
        return cuda_status(cudaGetLastError(), "k_gneb_project");
    }
    mj_status iterate(double* F, double* m, double* E, double* img, const GnebCtl* ctl) {
        mj_status e = images(F, m, E);
        if (e != MJ_OK) return e;
        const int nblk = static_cast<int>((X.n + 255) / 256);
        k_gneb_sums<<<dim3(nrep, nblk), 256, 0, s>>>(m, F, X, nrep, part, cnt, img, ctl);
        return cuda_status(cudaGetLastError(), "k_gneb_sums");
    }
};

}  // namespace
}  // namespace mj

using namespace mj;

extern "C" {

mj_status mj_gneb_path(mj_plan* plan, double* m, int32_t nimg, const mj_gneb_params* p, double* rx, double* ene,
                       double* dene, int64_t* iterations, double* max_force, int32_t* climbing, void* stream) {
    if (!plan || !m) return set_error(MJ_ERR_ARG, "bad GNEB arguments (no plan or path)");
    mj_status st = gneb_check(p, nimg, rx, ene, dene);
    if (st != MJ_OK) return st;
    // one magnetic atom per cell, as the reference's find_path requires
    // (GNEB/gneb_utils.f90:69, ERROR STOP for dim_mode /= 3)
    if (plan->nmag != 1) return set_error(MJ_ERR_UNSUPPORTED, "GNEB needs one magnetic atom per cell");
    const int64_t n = plan->N;
    const int64_t nblk = (n + 255) / 256;
    if (nblk > 65535) return set_error(MJ_ERR_UNSUPPORTED, "GNEB on a plan: at most 65535 x 256 spins per image");
    cudaSetDevice(plan->device);
    // the iterations are captured as a graph, which the legacy default stream
    // cannot hold: they run on the plan's own non-blocking stream, after the work
    // queued on `stream`
    if (!plan->cap_stream &&
        (st = cuda_status(cudaStreamCreateWithFlags(&plan->cap_stream, cudaStreamNonBlocking), "capture stream")) !=
            MJ_OK)
        return st;
    cudaStream_t s = plan->cap_stream;
    cudaEvent_t ready = nullptr;
    st = cuda_status(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "GNEB start");
    if (st == MJ_OK) st = cuda_status(cudaEventRecord(ready, static_cast<cudaStream_t>(stream)), "GNEB start");
    if (st == MJ_OK) st = cuda_status(cudaStreamWaitEvent(s, ready, 0), "GNEB start");
    PlanFields fl{plan, nimg, GnebIdx{n, 3 * n, n}, s, nullptr, nullptr};
    if (st == MJ_OK) st = cuda_status(cudaMalloc(&fl.part, sizeof(double) * 6 * nblk * nimg), "GNEB buffers");
    if (st == MJ_OK) st = cuda_status(cudaMalloc(&fl.cnt, sizeof(unsigned int) * nimg), "GNEB buffers");
    if (st == MJ_OK) st = cuda_status(cudaMemsetAsync(fl.cnt, 0, sizeof(unsigned int) * nimg, s), "GNEB buffers");
    // no per-kernel event records inside the captured iterations
    const bool prof = plan->prof_on;
    plan->prof_on = false;
    if (st == MJ_OK)
        st = gneb_relax(fl, m, nimg, fl.X, plan->num_sms, s, p, 32, rx, ene, dene, iterations, max_force, climbing);
    plan->prof_on = prof;
    const mj_status fin = cuda_status(cudaStreamSynchronize(s), "GNEB end");
    if (st == MJ_OK) st = fin;
    cudaFree(fl.part);
    cudaFree(fl.cnt);
    if (ready) cudaEventDestroy(ready);
    return st;
}

}  // extern "C"
