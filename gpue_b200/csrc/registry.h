// registry.h -- the compiled pass kernels, one pair (row, strided) per
// precision and line length, with the radix plan each was built for.
#pragma once

#include "pass.cuh"

namespace gpue {

enum Precision : int { PREC_F64 = 0, PREC_F32 = 1 };

struct PassKernel {
    int n;        // line length
    int ra, rb;   // radix plan (ra, ra) or (ra, rb, ra)
    int p;        // threads per line
    int ls;       // shared-memory line stride (elements per re/im array)
    int elem;     // bytes per complex element
    void (*row)(PassArgs);
    void (*col)(PassArgs);
};

// nullptr when the length has no compiled plan
const PassKernel* find_pass_kernel(int prec, int n);
// supported line lengths, ascending; returns the count
int supported_lengths(int prec, const int** out);

const PassKernel* pass_table_f32(int* count);
const PassKernel* pass_table_f64(int* count);

}  // namespace gpue
