// kernels_f32_b.cu -- complex64 pass kernels (the fused FP32 form), lengths >= 256.
//
// Plans per line length: radix sequence (RA, RA), (RA, RB, RA) or
// (RA, RB, RC, RA) and P threads per line.  E = N/P values per thread must be
// a multiple of every radix; the defaults keep E <= 16 where the length
// allows it and E = 12 or 20 for the radix-3 and radix-5 lengths (more
// resident warps, shorter straight-line code, fewer spills).  The
// first plan of a length is the default; the others (fewer threads per line,
// so a strided pass can take more lines per CTA and read whole 128-byte rows)
// are candidates for the autotuner.
#include "registry.h"

namespace gpue {

static const PassKernel kTable[] = {
    GPUE_PLAN(float, 256, 8, 4, 32),
    GPUE_PLAN(float, 256, 16, 0, 16),
    GPUE_PLAN(float, 320, 4, 20, 16),
    GPUE_PLAN4(float, 320, 4, 5, 4, 16, kMaxPassThreads, 2),
    GPUE_PLAN4(float, 384, 4, 6, 4, 32, kMaxPassThreads, 2),
    GPUE_PLAN(float, 384, 4, 24, 16),
    GPUE_PLAN(float, 512, 8, 8, 64),
    GPUE_PLAN(float, 512, 8, 8, 32),
    GPUE_PLAN4(float, 640, 4, 10, 4, 32, kMaxPassThreads, 2),
    GPUE_PLAN(float, 640, 8, 10, 16),
    GPUE_PLAN4(float, 768, 4, 12, 4, 64, kMaxPassThreads, 2),
    GPUE_PLAN(float, 768, 8, 12, 32),
    GPUE_PLAN(float, 1024, 16, 4, 64),
};

const PassKernel* pass_table_f32_b(int* count) {
    *count = (int)(sizeof(kTable) / sizeof(kTable[0]));
    return kTable;
}

}  // namespace gpue
