// Compile-time neighbour-offset tables of the lattices the tiled kernels
// specialise on.  Shared by the host (offset matching, coupling order) and the
// device (fully unrolled stencils with constant offsets).
#pragma once

namespace mj {

enum ShapeId { kShapeGeneric = 0, kShapeSquareNN = 1, kShapeTriNN = 2, kShapeTri3 = 3, kShapeSquare2 = 4 };

// square lattice, nearest neighbours (+-x, +-y): J + interfacial DMI
struct ShapeSquareNN {
    static constexpr int id = kShapeSquareNN;
    static constexpr int K = 4, R = 1;
    static constexpr int DX[K] = {1, -1, 0, 0};
    static constexpr int DY[K] = {0, 0, 1, -1};
    static constexpr int ISO[K] = {0, 0, 0, 0};
};

// square lattice, nearest + next-nearest (diagonal) neighbours
struct ShapeSquare2 {
    static constexpr int id = kShapeSquare2;
    static constexpr int K = 8, R = 1;
    static constexpr int DX[K] = {1, -1, 0, 0, 1, -1, 1, -1};
    static constexpr int DY[K] = {0, 0, 1, -1, 1, -1, -1, 1};
    static constexpr int ISO[K] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// triangular lattice (a1, a2 at 120 degrees), first shell: J1 + DMI
struct ShapeTriNN {
    static constexpr int id = kShapeTriNN;
    static constexpr int K = 6, R = 1;
    static constexpr int DX[K] = {1, -1, 0, 0, 1, -1};
    static constexpr int DY[K] = {0, 0, 1, -1, 1, -1};
    static constexpr int ISO[K] = {0, 0, 0, 0, 0, 0};
};

// triangular lattice, three shells: J1 + DMI (full tensors), J2 and J3 (isotropic)
struct ShapeTri3 {
    static constexpr int id = kShapeTri3;
    static constexpr int K = 18, R = 2;
    static constexpr int DX[K] = {1, -1, 0, 0, 1, -1, 1, -1, 2, -2, 1, -1, 2, -2, 0, 0, 2, -2};
    static constexpr int DY[K] = {0, 0, 1, -1, 1, -1, -1, 1, 1, -1, 2, -2, 0, 0, 2, -2, 2, -2};
    static constexpr int ISO[K] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
};

#ifdef __CUDACC__
#define MJ_HD __host__ __device__
#else
#define MJ_HD
#endif

template <class S>
MJ_HD constexpr int shape_col_ymin(int dx) {
    int m = 1 << 20;
    for (int k = 0; k < S::K; ++k)
        if (S::DX[k] == dx && S::DY[k] < m) m = S::DY[k];
    return m;
}
template <class S>
MJ_HD constexpr int shape_col_ymax(int dx) {
    int m = -(1 << 20);
    for (int k = 0; k < S::K; ++k)
        if (S::DX[k] == dx && S::DY[k] > m) m = S::DY[k];
    return m;
}

}  // namespace mj
