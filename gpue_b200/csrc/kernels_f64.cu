// kernels_f32.cu -- complex128 pass kernels (the plain FP64 form).
//
// One plan per line length: radix sequence (RA, RA) or (RA, RB, RA) and P
// threads per line, chosen for E = N/P <= 16 complex values per thread where
// the length allows it (more resident warps, shorter straight-line code).
#include "registry.h"

namespace gpue {

#define GPUE_PLAN(T, N, RA, RB, P)                                                        \
    PassKernel{N, RA, RB, P, LineFFT<T, N, RA, RB, P>::LS, (int)sizeof(cx<T>),            \
               &k_pass<T, N, RA, RB, P, false>, &k_pass<T, N, RA, RB, P, true>}

static const PassKernel kTableF64[] = {
    GPUE_PLAN(double, 16, 4, 0, 4),
    GPUE_PLAN(double, 32, 4, 2, 8),
    GPUE_PLAN(double, 64, 4, 4, 16),
    GPUE_PLAN(double, 96, 4, 6, 8),
    GPUE_PLAN(double, 128, 4, 8, 16),
    GPUE_PLAN(double, 160, 4, 10, 8),
    GPUE_PLAN(double, 192, 4, 12, 16),
    GPUE_PLAN(double, 256, 8, 4, 32),
    GPUE_PLAN(double, 320, 4, 20, 16),
    GPUE_PLAN(double, 384, 4, 24, 16),
    GPUE_PLAN(double, 512, 8, 8, 64),
    GPUE_PLAN(double, 640, 8, 10, 16),
    GPUE_PLAN(double, 768, 8, 12, 32),
    GPUE_PLAN(double, 1024, 16, 4, 64),
};

const PassKernel* pass_table_f64(int* count) {
    *count = (int)(sizeof(kTableF64) / sizeof(kTableF64[0]));
    return kTableF64;
}

}  // namespace gpue
