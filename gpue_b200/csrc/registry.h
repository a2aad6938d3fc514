// registry.h -- the compiled pass kernels, one pair (row, strided) per
// precision and line length, with the radix plan each was built for.
#pragma once

#include "pass.cuh"

namespace gpue {

enum Precision : int { PREC_F64 = 0, PREC_F32 = 1 };

struct PassKernel {
    int n;          // line length
    int ra, rb, rc; // radix plan (ra, ra), (ra, rb, ra) or (ra, rb, rc, ra)
    int p;          // threads per line
    int ls;         // shared-memory line stride (elements per re/im array)
    int elem;       // bytes per complex element
    int max_threads; // CTA size the kernels are compiled for
    void (*row)(PassArgs);
    void (*col)(PassArgs);
    void (*row_ext)(PassArgs);  // with table / expression factor forms
    void (*col_ext)(PassArgs);
    void (*row_batch)(const PassArgs*, const long*, int);  // independent solves at once
    void (*col_batch)(const PassArgs*, const long*, int);
};

// An XY-plane pass pair for 3D fields with nx = ny = n (plane.cuh): a cluster
// of cs CTAs of `threads` threads and `smem` bytes of dynamic shared memory
// per plane, persistent over the z-planes.
struct PlaneKernel {
    int n;
    int ra, rb, rc, p;  // the line FFT plan of both in-plane transforms
    int cs;             // CTAs per cluster
    int threads;
    int smem;
    void (*fwd)(PassArgs);  // rows [scale] V/2 Fx, columns Fy
    void (*inv)(PassArgs);  // rows Ix, columns Iy V/2 [norm]
};
// nullptr when no plane pass is compiled for (precision, n)
const PlaneKernel* find_plane_kernel(int prec, int n);

// The TMA z pass (tstream.cuh) for 3D fields with nz = n: tiles of 16
// x-columns, `threads` threads and `smem` bytes per CTA; a kernel taking
// (z-tile tensor map, unused tensor map, PassArgs, counters) (passed as void*
// here to keep cuda.h out).
struct ZPassKernel {
    int n;
    int ra, rb, rc, p;
    int threads;
    int smem;
    const void* fn;
};
const ZPassKernel* find_zpass_kernel(int prec, int n);

// The XY pass pair (tstream.cuh) for 3D fields with nx = ny = n: kernels
// taking (x-tile tensor map, y-tile tensor map, PassArgs, counters).
struct XYKernel {
    int n;
    int ra, rb, rc, p;
    int threads;
    int smem;
    const void* fwd;
    const void* inv;
};
const XYKernel* find_xy_kernel(int prec, int n);

// The persistent multi-size batched kernel (kernels_mega.cu): the tile body
// ("kind") of a line length and axis, -1 when the length is not covered;
// threads per line of a kind; the line stride of its plan; the kernel.
int mega_kind(int prec, int n, int axis);
int mega_threads_per_line(int kind);
int mega_plan_ls(int prec, int kind);
void* mega_kernel(int prec);

// The default plan for a length; nullptr when none is compiled
const PassKernel* find_pass_kernel(int prec, int n);
// All plans for a length, default first; returns how many (at most cap)
int find_pass_kernels(int prec, int n, const PassKernel** out, int cap);
// supported line lengths, ascending; returns the count
int supported_lengths(int prec, const int** out);

// The tables are split by length over translation units so they compile in
// parallel: _a holds lengths <= 192, _b lengths >= 256.
const PassKernel* pass_table_f32_a(int* count);
const PassKernel* pass_table_f32_b(int* count);
const PassKernel* pass_table_f64_a(int* count);
const PassKernel* pass_table_f64_b(int* count);

#define GPUE_PLAN4(T, N, RA, RB, RC, P, MAXT, MINB)                                        \
    PassKernel{N, RA, RB, RC, P, LineFFT<T, N, RA, RB, P, RC>::LS, (int)sizeof(cx<T>), MAXT,   \
               &k_pass<T, N, RA, RB, P, false, false, RC, MAXT, MINB>,                       \
               &k_pass<T, N, RA, RB, P, true, false, RC, MAXT, MINB>,                        \
               &k_pass<T, N, RA, RB, P, false, true, RC, MAXT, MINB>,                        \
               &k_pass<T, N, RA, RB, P, true, true, RC, MAXT, MINB>,                         \
               &k_pass_batch<T, N, RA, RB, P, false, RC, MAXT, MINB>,                        \
               &k_pass_batch<T, N, RA, RB, P, true, RC, MAXT, MINB>}
#define GPUE_PLAN(T, N, RA, RB, P) GPUE_PLAN4(T, N, RA, RB, 0, P, kMaxPassThreads, 2)

}  // namespace gpue
