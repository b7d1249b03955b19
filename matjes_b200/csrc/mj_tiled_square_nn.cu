// Tiled kernels of one lattice shape (ShapeSquareNN); see mj_tiled_impl.cuh.
#include "mj_tiled_impl.cuh"

namespace mj {
mj_status launch_tiled_square_nn(mj_plan* p, int pass, const DynCoef& C, const double* ms, const double* mn, double* out,
                         double* aux, double* aux2, DipView Hd, double* E_out, uint32_t step, cudaStream_t s,
                         int emode, int ty0, int nty) {
    return launch_tiled_shape<ShapeSquareNN>(p, pass, C, ms, mn, out, aux, aux2, Hd, E_out, step, s, emode, ty0, nty);
}
mj_status launch_sib_fused_square_nn(mj_plan* p, const DynCoef& C, double* m, double* draw, double* E_out, uint32_t step,
                         cudaStream_t s) {
    return launch_sib_fused_shape<ShapeSquareNN>(p, C, m, draw, E_out, step, s);
}
mj_status launch_gneb_images_square_nn(mj_plan* p, const double* m, double* F, double* partials, int nimg,
                         int64_t* tiles, cudaStream_t s) {
    return launch_gneb_images_shape<ShapeSquareNN>(p, m, F, partials, nimg, tiles, s);
}
}  // namespace mj
