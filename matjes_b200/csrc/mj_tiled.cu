// Dispatch of the tiled kernels to the translation unit of the plan's shape,
// and the self-test of their bounded-wait failure path.
#include "mj_internal.hpp"
#include "mj_shapes.hpp"
#include "mj_tiled_impl.cuh"

namespace mj {
namespace {

// One block arms an mbarrier for 16 bytes that no copy delivers (no TMA is
// issued, so nothing is in flight), gives up after `polls` polls through the
// same bounded wait as k_tiled, and records the timeout as k_tiled does.
__global__ void k_selftest_timeout(uint32_t polls, int* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        mbar_expect_tx(&bar, 16u);
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0u, polls);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(status, kStatusTimeout);
    }
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&bar)) : "memory");
}

}  // namespace

int64_t tiled_energy_blocks(const mj_plan* p) {
    const int v = (p->tile_variant >= 0 && p->tile_variant < kTiledVariants) ? p->tile_variant : 0;
    const int ty = kTiledVariantTY[v];
    return static_cast<int64_t>((p->sp.L[0] + 31) / 32) * ((p->sp.L[1] + ty - 1) / ty) * p->sp.L[2];
}

int64_t sched_words(const mj_plan* p) {
    int min_ty = kTiledVariantTY[0];
    for (int v = 1; v < kTiledVariants; ++v) min_ty = std::min(min_ty, kTiledVariantTY[v]);
    return 2 + static_cast<int64_t>((p->sp.L[1] + min_ty - 1) / min_ty) * p->sp.L[2];
}

mj_status launch_sib_fused(mj_plan* p, const DynCoef& C, double* m, double* draw, double* E_out, uint32_t step,
                           cudaStream_t s) {
    if (!p->d_sched) return set_error(MJ_ERR_ARG, "plan has no fused-step scheduler");
    switch (p->sp.shape) {
        case kShapeSquareNN: return launch_sib_fused_square_nn(p, C, m, draw, E_out, step, s);
        case kShapeSquare2: return launch_sib_fused_square2(p, C, m, draw, E_out, step, s);
        case kShapeTriNN: return launch_sib_fused_tri_nn(p, C, m, draw, E_out, step, s);
        case kShapeTri3: return launch_sib_fused_tri3(p, C, m, draw, E_out, step, s);
        default: return set_error(MJ_ERR_ARG, "no tiled kernel for this stencil shape");
    }
}

mj_status launch_gneb_images(mj_plan* p, const double* m, double* F, double* partials, int nimg,
                             int64_t* tiles_per_image, cudaStream_t s) {
    switch (p->sp.shape) {
        case kShapeSquareNN: return launch_gneb_images_square_nn(p, m, F, partials, nimg, tiles_per_image, s);
        case kShapeSquare2: return launch_gneb_images_square2(p, m, F, partials, nimg, tiles_per_image, s);
        case kShapeTriNN: return launch_gneb_images_tri_nn(p, m, F, partials, nimg, tiles_per_image, s);
        case kShapeTri3: return launch_gneb_images_tri3(p, m, F, partials, nimg, tiles_per_image, s);
        default: return set_error(MJ_ERR_ARG, "no tiled kernel for this stencil shape");
    }
}

int tiled_tile_rows(const mj_plan* p) {
    const int v = (p->tile_variant >= 0 && p->tile_variant < kTiledVariants) ? p->tile_variant : 0;
    const int ty = kTiledVariantTY[v];
    return (p->sp.L[1] + ty - 1) / ty;
}

mj_status launch_tiled(mj_plan* p, int pass, const DynCoef& C, const double* ms, const double* mn, double* out,
                       double* aux, double* aux2, DipView Hd, double* E_out, uint32_t step, cudaStream_t s,
                       int emode, int ty0, int nty) {
    switch (p->sp.shape) {
        case kShapeSquareNN:
            return launch_tiled_square_nn(p, pass, C, ms, mn, out, aux, aux2, Hd, E_out, step, s, emode, ty0, nty);
        case kShapeSquare2:
            return launch_tiled_square2(p, pass, C, ms, mn, out, aux, aux2, Hd, E_out, step, s, emode, ty0, nty);
        case kShapeTriNN:
            return launch_tiled_tri_nn(p, pass, C, ms, mn, out, aux, aux2, Hd, E_out, step, s, emode, ty0, nty);
        case kShapeTri3:
            return launch_tiled_tri3(p, pass, C, ms, mn, out, aux, aux2, Hd, E_out, step, s, emode, ty0, nty);
        default: return set_error(MJ_ERR_ARG, "no tiled kernel for this stencil shape");
    }
}

}  // namespace mj

using namespace mj;

extern "C" mj_status mj_plan_selftest_timeout(mj_plan* plan, uint32_t polls, void* stream) {
    if (!plan) return set_error(MJ_ERR_ARG, "null plan");
    if (polls < 1 || polls > (1u << 16)) return set_error(MJ_ERR_ARG, "polls must be in [1, 65536]");
    cudaSetDevice(plan->device);
    k_selftest_timeout<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(polls, plan->d_status);
    return cuda_status(cudaGetLastError(), "k_selftest_timeout");
}
