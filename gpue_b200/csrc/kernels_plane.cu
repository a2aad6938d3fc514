// kernels_plane.cu -- the complex64 XY-plane pass kernels (plane.cuh) for the
// 3D step, one forward/inverse pair per in-plane length, each with the line
// length's default radix plan.
#include "registry.h"
#include "plane.cuh"

namespace gpue {

#define GPUE_PLANE(T, N, RA, RB, RC, P)                                                     \
    PlaneKernel{N, RA, RB, RC, P, PlaneShape<T, N, RA, RB, P, RC, 16>::CS,                   \
                PlaneShape<T, N, RA, RB, P, RC, 16>::THREADS,                                \
                (int)PlaneShape<T, N, RA, RB, P, RC, 16>::SMEM,                              \
                &k_plane<T, N, RA, RB, P, RC, 16, false>,                                    \
                &k_plane<T, N, RA, RB, P, RC, 16, true>}

static const PlaneKernel kPlanesF32[] = {
    GPUE_PLANE(float, 64, 4, 4, 0, 16),
    GPUE_PLANE(float, 96, 4, 6, 0, 8),
    GPUE_PLANE(float, 128, 4, 8, 0, 16),
    GPUE_PLANE(float, 160, 4, 10, 0, 8),
    GPUE_PLANE(float, 192, 4, 12, 0, 16),
    GPUE_PLANE(float, 256, 16, 0, 0, 16),
};

const PlaneKernel* find_plane_kernel(int prec, int n) {
    if (prec != PREC_F32) return nullptr;
    for (const PlaneKernel& k : kPlanesF32)
        if (k.n == n) return &k;
    return nullptr;
}

}  // namespace gpue
