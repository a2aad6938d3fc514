// kernels_plane.cu -- the complex64 pass kernels of the 3D step beyond the
// line passes: the cluster XY-plane passes (plane.cuh) and the TMA tile-stream
// XY and z passes (tstream.cuh), per length with the line length's default
// radix plan.
#include "registry.h"
#include "plane.cuh"
#include "tstream.cuh"

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

#define GPUE_ZPASS(T, N, RA, RB, RC, P)                                                     \
    ZPassKernel{N, RA, RB, RC, P, TSShape<T, N, RA, RB, P, RC>::THREADS,                     \
                (int)TSShape<T, N, RA, RB, P, RC>::SMEM,                                     \
                (const void*)&k_tstream<T, N, RA, RB, P, RC, TS_Z>}

static const ZPassKernel kZPassF32[] = {
    GPUE_ZPASS(float, 64, 4, 4, 0, 16),
    GPUE_ZPASS(float, 96, 4, 6, 0, 8),
    GPUE_ZPASS(float, 128, 4, 8, 0, 16),
    GPUE_ZPASS(float, 160, 4, 10, 0, 8),
    GPUE_ZPASS(float, 192, 4, 12, 0, 16),
    GPUE_ZPASS(float, 256, 16, 0, 0, 16),
};

#define GPUE_XY(T, N, RA, RB, RC, P)                                                        \
    XYKernel{N, RA, RB, RC, P, TSShape<T, N, RA, RB, P, RC>::THREADS,                        \
             (int)TSShape<T, N, RA, RB, P, RC>::SMEM,                                        \
             (const void*)&k_tstream<T, N, RA, RB, P, RC, TS_XY_FWD>,                        \
             (const void*)&k_tstream<T, N, RA, RB, P, RC, TS_XY_INV>}

static const XYKernel kXYF32[] = {
    GPUE_XY(float, 64, 4, 4, 0, 16),
    GPUE_XY(float, 96, 4, 6, 0, 8),
    GPUE_XY(float, 128, 4, 8, 0, 16),
    GPUE_XY(float, 160, 4, 10, 0, 8),
    GPUE_XY(float, 192, 4, 12, 0, 16),
    GPUE_XY(float, 256, 16, 0, 0, 16),
};

const XYKernel* find_xy_kernel(int prec, int n) {
    if (prec != PREC_F32) return nullptr;
    for (const XYKernel& k : kXYF32)
        if (k.n == n) return &k;
    return nullptr;
}

const ZPassKernel* find_zpass_kernel(int prec, int n) {
    if (prec != PREC_F32) return nullptr;
    for (const ZPassKernel& k : kZPassF32)
        if (k.n == n) return &k;
    return nullptr;
}

const PlaneKernel* find_plane_kernel(int prec, int n) {
    if (prec != PREC_F32) return nullptr;
    for (const PlaneKernel& k : kPlanesF32)
        if (k.n == n) return &k;
    return nullptr;
}

}  // namespace gpue
