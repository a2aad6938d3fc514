// kernels_f32_a.cu -- complex64 pass kernels (the fused FP32 form), lengths <= 192.
//
// One plan per line length: radix sequence (RA, RA) or (RA, RB, RA) and P
// threads per line, chosen for E = N/P <= 16 complex values per thread where
// the length allows it (more resident warps, shorter straight-line code).
// Their P <= 16 already lets a strided pass read whole 128-byte rows.
#include "registry.h"

namespace gpue {

static const PassKernel kTable[] = {
    GPUE_PLAN(float, 16, 4, 0, 4),
    GPUE_PLAN(float, 32, 4, 2, 8),
    GPUE_PLAN(float, 64, 4, 4, 16),
    GPUE_PLAN(float, 96, 4, 6, 8),
    GPUE_PLAN(float, 128, 4, 8, 16),
    GPUE_PLAN(float, 160, 4, 10, 8),
    GPUE_PLAN(float, 192, 4, 12, 16),
};

const PassKernel* pass_table_f32_a(int* count) {
    *count = (int)(sizeof(kTable) / sizeof(kTable[0]));
    return kTable;
}

}  // namespace gpue
