// kernels_f32.cu -- complex64 pass kernels (the fused FP32 form).
//
// One plan per line length: radix sequence (RA, RA) or (RA, RB, RA) and P
// threads per line, chosen for E = N/P <= 16 complex values per thread where
// the length allows it (more resident warps, shorter straight-line code).
#include "registry.h"

namespace gpue {

#define GPUE_PLAN(T, N, RA, RB, P)                                                        \
    PassKernel{N, RA, RB, P, LineFFT<T, N, RA, RB, P>::LS, (int)sizeof(cx<T>),            \
               &k_pass<T, N, RA, RB, P, false>, &k_pass<T, N, RA, RB, P, true>}

static const PassKernel kTableF32[] = {
    GPUE_PLAN(float, 16, 4, 0, 4),
    GPUE_PLAN(float, 32, 4, 2, 8),
    GPUE_PLAN(float, 64, 4, 4, 16),
    GPUE_PLAN(float, 96, 4, 6, 8),
    GPUE_PLAN(float, 128, 4, 8, 16),
    GPUE_PLAN(float, 160, 4, 10, 8),
    GPUE_PLAN(float, 192, 4, 12, 16),
    GPUE_PLAN(float, 256, 8, 4, 32),
    GPUE_PLAN(float, 320, 4, 20, 16),
    GPUE_PLAN(float, 384, 4, 24, 16),
    GPUE_PLAN(float, 512, 8, 8, 64),
    GPUE_PLAN(float, 640, 8, 10, 16),
    GPUE_PLAN(float, 768, 8, 12, 32),
    GPUE_PLAN(float, 1024, 16, 4, 64),
};

const PassKernel* pass_table_f32(int* count) {
    *count = (int)(sizeof(kTableF32) / sizeof(kTableF32[0]));
    return kTableF32;
}

}  // namespace gpue
