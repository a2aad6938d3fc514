// kernels_f32.cu -- complex64 pass kernels (the fused FP32 form).
#include "registry.h"

namespace gpue {

#define GPUE_PLAN(T, N, RA, RB, P)                                                        \
    PassKernel{N, RA, RB, P, LineFFT<T, N, RA, RB, P>::LS, (int)sizeof(cx<T>),            \
               &k_pass<T, N, RA, RB, P, false>, &k_pass<T, N, RA, RB, P, true>}

static const PassKernel kTableF32[] = {
    GPUE_PLAN(float, 16, 4, 0, 4),
    GPUE_PLAN(float, 32, 4, 2, 8),
    GPUE_PLAN(float, 64, 8, 0, 8),
    GPUE_PLAN(float, 96, 4, 6, 8),
    GPUE_PLAN(float, 128, 8, 2, 16),
    GPUE_PLAN(float, 160, 4, 10, 8),
    GPUE_PLAN(float, 192, 4, 12, 16),
    GPUE_PLAN(float, 256, 16, 0, 16),
    GPUE_PLAN(float, 320, 4, 20, 16),
    GPUE_PLAN(float, 384, 4, 24, 16),
    GPUE_PLAN(float, 512, 8, 8, 32),
    GPUE_PLAN(float, 640, 8, 10, 16),
    GPUE_PLAN(float, 768, 8, 12, 32),
    GPUE_PLAN(float, 1024, 32, 0, 32),
};

const PassKernel* pass_table_f32(int* count) {
    *count = (int)(sizeof(kTableF32) / sizeof(kTableF32[0]));
    return kTableF32;
}

}  // namespace gpue
