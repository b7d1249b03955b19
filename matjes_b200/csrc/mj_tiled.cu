// Dispatch of the tiled kernels to the translation unit of the plan's shape.
#include "mj_internal.hpp"
#include "mj_shapes.hpp"

namespace mj {

int64_t tiled_energy_blocks(const mj_plan* p) {
    const int v = (p->tile_variant >= 0 && p->tile_variant < kTiledVariants) ? p->tile_variant : 0;
    const int ty = kTiledVariantTY[v];
    return static_cast<int64_t>((p->sp.L[0] + 31) / 32) * ((p->sp.L[1] + ty - 1) / ty) * p->sp.L[2];
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
