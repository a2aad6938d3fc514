// kernels_f64_a.cu -- complex128 pass kernels (the plain FP64 form), lengths <= 192.
//
// One plan per line length: radix sequence (RA, RA) or (RA, RB, RA) and P
// threads per line, chosen for E = N/P <= 16 complex values per thread where
// the length allows it (more resident warps, shorter straight-line code).
// Their P <= 16 already lets a strided pass read whole 128-byte rows.
#include "registry.h"

namespace gpue {

static const PassKernel kTable[] = {
    GPUE_PLAN(double, 16, 4, 0, 4),
    GPUE_PLAN(double, 32, 4, 2, 8),
    GPUE_PLAN(double, 64, 4, 4, 16),
    GPUE_PLAN(double, 96, 4, 6, 8),
    GPUE_PLAN(double, 128, 4, 8, 16),
    GPUE_PLAN(double, 160, 4, 10, 8),
    GPUE_PLAN(double, 192, 4, 12, 16),
};

const PassKernel* pass_table_f64_a(int* count) {
    *count = (int)(sizeof(kTable) / sizeof(kTable[0]));
    return kTable;
}

}  // namespace gpue
