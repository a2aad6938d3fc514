// noalloc.cu -- sum |psi|^2 dV of a caller-owned device wavefunction with no
// device memory allocated by the library at any point.
//
// Some callers of this library cannot allocate device memory when they want a
// norm: a serving process that reserved its whole HBM budget up front and
// hands out fixed slices, or a host thread running next to another
// framework's caching allocator that already holds the free memory.  For
// them gpue_norm_noalloc() works on a wavefunction they own and writes the
// result to memory they own.  The cross-block reduction scratch lives in one
// file-scope __device__ array (kNaBytes below) that every GPU loading the
// library holds until the process exits.
//
// The array's name is only a host-side stand-in in host code; the device
// address comes from cudaGetSymbolAddress, asked on every call with the
// caller's device current (a lookup that allocates nothing), so a device
// whose primary context was reset in between gets its new address.  The
// first call on a device also loads the library's device code there, so make
// it before any stream capture.  Every call on a device shares the one array
// and it keeps the previous call's contents: the arrival counter is cleared
// before each launch, and calls whose kernels overlap on the GPU (different
// streams, no ordering between them) race on the array.

#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/gpue_b200.h"
#include "pass.cuh"

namespace {

using gpue::cx;
using gpue::KSum;

constexpr int kNaThreads = 256;
constexpr int kNaPerBlock = 4096;      // points reduced by one block
constexpr int kNaMaxBlocks = 65536;    // partial sums the scratch holds
constexpr long long kNaMaxPoints = (long long)kNaMaxBlocks * kNaPerBlock;  // 2^28

struct NaScratch {
    double2 partials[kNaMaxBlocks];  // 1 MiB
    unsigned counter;                // blocks finished; must start at 0
    unsigned pad[63];
};
constexpr size_t kNaBytes = sizeof(NaScratch);

static __device__ __align__(256) NaScratch g_na_scratch;

// This entry point has no context to hold a message, so failures are reported
// by the status code and one line on stderr.
gpue_status na_fail(gpue_status st, const char* msg) {
    fprintf(stderr, "%s\n", msg);
    return st;
}

template <typename T>
__global__ void __launch_bounds__(kNaThreads) k_norm_noalloc(const void* psi_, long long n,
                                                             double dV, double* out,
                                                             NaScratch* s) {
    __shared__ double scratch[2 * (kNaThreads / 32)];
    __shared__ unsigned last;
    const cx<T>* psi = reinterpret_cast<const cx<T>*>(psi_);
    const long long b0 = (long long)blockIdx.x * kNaPerBlock;
    KSum acc{0.0, 0.0};
    for (int i = threadIdx.x; i < kNaPerBlock; i += kNaThreads) {
        const long long g = b0 + i;
        if (g < n) {
            const cx<T> v = psi[g];
            acc.add((double)v.x * v.x + (double)v.y * v.y);
        }
    }
    acc = gpue::block_reduce(acc, scratch);
    if (threadIdx.x == 0) {
        s->partials[blockIdx.x] = make_double2(acc.s, acc.c);
        __threadfence();
        last = (atomicAdd(&s->counter, 1u) == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (last) {
        __threadfence();
        KSum t{0.0, 0.0};
        for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
            const double2 p = __ldcg(&s->partials[i]);
            t.merge(p.x, p.y);
        }
        __syncthreads();
        t = gpue::block_reduce(t, scratch);
        if (threadIdx.x == 0) {
            out[0] = (t.s + t.c) * dV;
            s->counter = 0u;
        }
    }
}

}  // namespace

extern "C" gpue_status gpue_norm_noalloc(const void* psi, int32_t dtype, int64_t npoints,
                                         double dV, double* out, void* stream) {
    if (!psi || !out || (dtype != GPUE_C128 && dtype != GPUE_C64))
        return na_fail(GPUE_ERR_INVALID_ARG, "gpue_norm_noalloc: null pointer or bad dtype");
    if (npoints < 1 || npoints > kNaMaxPoints) {
        char m[160];
        snprintf(m, sizeof m,
                 "gpue_norm_noalloc: %lld points is outside 1..%lld, the most its "
                 "fixed %zu-byte device scratch covers",
                 (long long)npoints, kNaMaxPoints, kNaBytes);
        return na_fail(GPUE_ERR_INVALID_ARG, m);
    }
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_na_scratch) != cudaSuccess || !p)
        return na_fail(GPUE_ERR_CUDA, "gpue_norm_noalloc: cudaGetSymbolAddress failed");
    NaScratch* sp = static_cast<NaScratch*>(p);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(&sp->counter, 0, sizeof(unsigned), s) != cudaSuccess)
        return na_fail(GPUE_ERR_CUDA, "gpue_norm_noalloc: clearing the counter failed");
    const int blocks = (int)((npoints + kNaPerBlock - 1) / kNaPerBlock);
    if (dtype == GPUE_C128)
        k_norm_noalloc<double><<<blocks, kNaThreads, 0, s>>>(psi, npoints, dV, out, sp);
    else
        k_norm_noalloc<float><<<blocks, kNaThreads, 0, s>>>(psi, npoints, dV, out, sp);
    if (cudaGetLastError() != cudaSuccess)
        return na_fail(GPUE_ERR_CUDA, "gpue_norm_noalloc: kernel launch failed");
    return GPUE_OK;
}
