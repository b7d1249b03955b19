// GNEB path relaxation on any plan: find_path of GNEB/gneb_utils.f90:19-240
// with the field of every image from the plan's own field kernels, so the path
// may live on any lattice of one magnetic atom per cell a plan holds (tiled and
// generic stencils, ELL couplings, open boundaries, 3D films) and the images see
// every term of the plan's Hamiltonian, the FFT dipolar term included, as
// get_eff_field and H%energy give them to the reference's GNEB (:77-81,
// :154-157).  The path is nimg images of the plan's N spins in one device
// array, image r the SoA block x[N] | y[N] | z[N] at 3 N r.
//
// The images' fields: on a tiled plan without the dipolar term one launch over
// all images (launch_gneb_images: blockIdx.z runs over image and layer, a 5D
// TMA map over the path) that also projects the field on each spin's tangent
// plane and leaves per tile the six path sums and the energy, then
// k_gneb_tile_sums adds the tiles of every image in tile order; otherwise per
// image one field launch (launch_field), the images side by side on forked
// streams unless the dipolar term's FFT grid is shared, then k_gneb_sums
// (projection, the six path sums and, for side-by-side images, the energy of
// every image) or, for the dipolar term's one-by-one launches that reduce
// their energies themselves, k_gneb_project outside the iterations.  The rest of
// the relaxation is mj_gneb.cuh's, shared with the replica batch.
#include <algorithm>
#include <cstring>

#include "mj_gneb.cuh"
#include "mj_internal.hpp"

namespace mj {
namespace {

// Per image (r = blockIdx.x): its T tile partials of the fused GNEB image pass
// (partials[q nb + r T + t], q = the six path sums, then the energy) added in
// tile order, warp q for quantity q, into img[q nrep + r] and E[r].
__global__ void __launch_bounds__(256) k_gneb_tile_sums(const double* __restrict__ part, int T, int64_t nb, int nrep,
                                                        double* img, double* E, const GnebCtl* ctl) {
    if (ctl && ctl->done) return;
    const int r = blockIdx.x;
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    if (q >= 7) return;
    const double* pq = part + q * nb + static_cast<int64_t>(r) * T;
    double v = 0.0;
    for (int t = lane; t < T; t += 32) v += pq[t];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) {
        if (q < 6) img[q * nrep + r] = v;
        else E[r] = v;
    }
}

// The field of the images for gneb_relax.  Without the dipolar term the images'
// field launches share no scratch (no total energy asked, per-site energies
// into their own slices): they run side by side on kSide forked streams, and
// k_gneb_sums sums each image's site energies with its path sums.  With the
// dipolar term (one padded FFT grid per plan) they run one after another, each
// reducing its own total energy.
struct PlanFields {
    static constexpr int kSide = 8;
    mj_plan* p;
    int nrep;
    GnebIdx X;
    cudaStream_t s;
    bool concurrent;
    bool tiled = false;           // the fused GNEB image pass of a tiled plan (set by setup)
    int64_t tiles = 0;            // its tiles per image
    double* part = nullptr;       // partials: 7 per (image, block or tile)
    unsigned int* cnt = nullptr;  // last-block counters, one per image
    double* esite = nullptr;      // per-site energies, image r at [r N, (r + 1) N) (concurrent form)
    double* img0 = nullptr;       // path sums of the calls outside the iterations (unused)
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kSide] = {};

    mj_status setup(int64_t nblk) {
        tiled = concurrent && p->is_stencil && p->sp.shape != 0;
        const int64_t nper = tiled ? std::max(nblk, tiled_energy_blocks(p)) : nblk;
        mj_status st = cuda_status(cudaMalloc(&part, sizeof(double) * 7 * nper * nrep), "GNEB buffers");
        if (st == MJ_OK) st = cuda_status(cudaMalloc(&cnt, sizeof(unsigned int) * nrep), "GNEB buffers");
        if (st == MJ_OK) st = cuda_status(cudaMalloc(&img0, sizeof(double) * 6 * nrep), "GNEB buffers");
        if (st == MJ_OK) st = cuda_status(cudaMemsetAsync(cnt, 0, sizeof(unsigned int) * nrep, s), "GNEB buffers");
        if (st != MJ_OK || !concurrent || tiled) return st;
        st = cuda_status(cudaMalloc(&esite, sizeof(double) * X.n * nrep), "GNEB buffers");
        if (st == MJ_OK) st = cuda_status(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "GNEB events");
        for (int k = 0; k < kSide && st == MJ_OK; ++k) {
            st = cuda_status(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking), "GNEB streams");
            if (st == MJ_OK) st = cuda_status(cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming), "GNEB events");
        }
        return st;
    }
    void release() {
        for (int k = 0; k < kSide; ++k) {
            if (side[k]) cudaStreamDestroy(side[k]);
            if (join[k]) cudaEventDestroy(join[k]);
        }
        if (fork) cudaEventDestroy(fork);
        for (double* b : {part, esite, img0}) cudaFree(b);
        cudaFree(cnt);
    }
    mj_status images(double* F, const double* m, double* E) {
        if (!concurrent) {
            for (int r = 0; r < nrep; ++r) {
                const int64_t o = static_cast<int64_t>(r) * X.is;
                mj_status e = launch_field(p, m + o, F + o, nullptr, E + r, s);
                if (e != MJ_OK) return e;
            }
            return MJ_OK;
        }
        const int nside = std::min(kSide, nrep);
        mj_status e = cuda_status(cudaEventRecord(fork, s), "GNEB fork");
        for (int k = 0; k < nside && e == MJ_OK; ++k) e = cuda_status(cudaStreamWaitEvent(side[k], fork, 0), "GNEB fork");
        for (int r = 0; r < nrep && e == MJ_OK; ++r) {
            const int64_t o = static_cast<int64_t>(r) * X.is;
            e = launch_field(p, m + o, F + o, esite + r * X.n, nullptr, side[r % nside]);
        }
        // the forked streams join the main one even after a failed launch
        for (int k = 0; k < nside; ++k) {
            const mj_status j = cuda_status(cudaEventRecord(join[k], side[k]), "GNEB join");
            const mj_status w = j == MJ_OK ? cuda_status(cudaStreamWaitEvent(s, join[k], 0), "GNEB join") : j;
            if (e == MJ_OK) e = w;
        }
        return e;
    }
    mj_status sums(double* F, double* m, double* E, double* img, const GnebCtl* ctl) {
        constexpr int kSpt = 4;  // sites per thread
        const int nblk = static_cast<int>((X.n + 256 * kSpt - 1) / (256 * kSpt));
        k_gneb_sums<kSpt><<<dim3(nrep, nblk), 256, 0, s>>>(m, F, X, nrep, concurrent ? esite : nullptr, E, part, cnt,
                                                           img, ctl);
        return cuda_status(cudaGetLastError(), "k_gneb_sums");
    }
    // tiled plans: one launch over all images (image r = blockIdx.z's image) with
    // the projection and the tiles' path sums, then the sums of every image
    mj_status gneb_tiled(double* F, const double* m, double* E, double* img, const GnebCtl* ctl) {
        const int rec = prof_begin(p, "k_gneb_images", s);
        mj_status e = launch_gneb_images(p, m, F, part, nrep, &tiles, s);
        prof_end(p, rec, s);
        if (e != MJ_OK) return e;
        k_gneb_tile_sums<<<nrep, 7 * 32, 0, s>>>(part, static_cast<int>(tiles), tiles * nrep, nrep, img, E, ctl);
        return cuda_status(cudaGetLastError(), "k_gneb_tile_sums");
    }
    mj_status field(double* F, double* m, double* E) {
        if (tiled) return gneb_tiled(F, m, E, img0, nullptr);
        mj_status e = images(F, m, E);
        if (e != MJ_OK) return e;
        if (concurrent) return sums(F, m, E, img0, nullptr);
        const int nblk = static_cast<int>((X.n + 255) / 256);
        k_gneb_project<<<dim3(nblk, nrep), 256, 0, s>>>(F, m, X);
        return cuda_status(cudaGetLastError(), "k_gneb_project");
    }
    mj_status iterate(double* F, double* m, double* E, double* img, const GnebCtl* ctl) {
        if (tiled) return gneb_tiled(F, m, E, img, ctl);
        mj_status e = images(F, m, E);
        if (e != MJ_OK) return e;
        return sums(F, m, E, img, ctl);
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
    PlanFields fl{plan, nimg, GnebIdx{n, 3 * n, n}, s, !plan->dip_on};
    if (st == MJ_OK) st = fl.setup(nblk);
    // no per-kernel event records inside the captured iterations
    const bool prof = plan->prof_on;
    plan->prof_on = false;
    if (st == MJ_OK)
        st = gneb_relax(fl, m, nimg, fl.X, plan->num_sms, s, p, 32, rx, ene, dene, iterations, max_force, climbing);
    plan->prof_on = prof;
    const mj_status fin = cuda_status(cudaStreamSynchronize(s), "GNEB end");
    if (st == MJ_OK) st = fin;
    // an image field launch whose bounded wait gave up left that image's forces
    // unfinished: the whole path is invalid
    int word = 0;
    if (st == MJ_OK)
        st = cuda_status(cudaMemcpy(&word, plan->d_status, sizeof(int), cudaMemcpyDeviceToHost), "GNEB status");
    if (st == MJ_OK) st = status_from_word(plan, word);
    fl.release();
    if (ready) cudaEventDestroy(ready);
    return st;
}

}  // extern "C"
