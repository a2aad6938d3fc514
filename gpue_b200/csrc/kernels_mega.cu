// kernels_mega.cu -- the persistent batched-run kernel (batch_mega.cuh) for
// both precisions, over the default plans of the line lengths 64 to 512.
#include "batch_mega.cuh"
#include "registry.h"

namespace gpue {

namespace {

// (length, radix plan, threads per line) of each tile body, in kind order
struct MegaPlan {
    int n, ra, rb, rc, p;
};
// (lengths whose default plan holds at most 12 values per thread: the longer
// bodies would raise the whole kernel's register spills)
constexpr MegaPlan kMegaPlans[] = {
    {64, 4, 4, 0, 16},   {128, 4, 8, 0, 16}, {192, 4, 12, 0, 16},
    {256, 8, 4, 0, 32},  {384, 4, 6, 4, 32}, {512, 8, 8, 0, 64},
};
constexpr int kMegaPlanCount = sizeof(kMegaPlans) / sizeof(kMegaPlans[0]);

template <typename T, int K>
__device__ __forceinline__ KSum mega_tile(const PassArgs& a, long tile, unsigned char* smem,
                                          bool strided) {
    constexpr MegaPlan m = kMegaPlans[K];
    if (strided)
        return pass_tiles<T, m.n, m.ra, m.rb, m.p, true, false, m.rc>(a, tile, a.ntiles, smem);
    return pass_tiles<T, m.n, m.ra, m.rb, m.p, false, false, m.rc>(a, tile, a.ntiles, smem);
}

template <typename T>
__device__ __forceinline__ KSum mega_dispatch(int kind, const PassArgs& a, long tile,
                                              unsigned char* smem) {
    const bool s = kind & 1;
    switch (kind >> 1) {
        case 0: return mega_tile<T, 0>(a, tile, smem, s);
        case 1: return mega_tile<T, 1>(a, tile, smem, s);
        case 2: return mega_tile<T, 2>(a, tile, smem, s);
        case 3: return mega_tile<T, 3>(a, tile, smem, s);
        case 4: return mega_tile<T, 4>(a, tile, smem, s);
        default: return mega_tile<T, 5>(a, tile, smem, s);
    }
}

template <typename T>
__global__ void __launch_bounds__(kMegaThreads, 2) k_batch_mega(const MegaArgs m) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long s_ticket;
    __shared__ int s_pass;
    for (;;) {
        if (threadIdx.x == 0) {
            const long t = (long)atomicAdd(m.ticket, 1ull);
            int pi = -1;
            if (t < m.total) {
                pi = m.item_pass[t];
                // wait until the pass before this one (same solve) is complete
                const int dep = m.passes[pi].dep;
                if (dep >= 0) {
                    const int need = m.passes[dep].nitems;
                    const volatile int* d = m.done + dep;
                    unsigned polls = 0;
                    while (*d < need) {
                        if (++polls >= kMegaWaitPolls) {
                            atomicExch(m.err, 1);
                            break;
                        }
                        __nanosleep(64);
                    }
                    __threadfence();
                }
            }
            s_ticket = t;
            s_pass = pi;
        }
        __syncthreads();
        const long t = s_ticket;
        const int pi = s_pass;
        __syncthreads();  // both read before thread 0 writes them again
        if (pi < 0) break;
        const MegaPass& p = m.passes[pi];
        const PassArgs& a = m.args[p.args];
        if (!(a.active && *a.active == 0)) {
            const long first = (t - p.start) * p.chunk;
            const long last = first + p.chunk < p.ntiles ? first + p.chunk : p.ntiles;
            for (long tile = first; tile < last; ++tile) {
                KSum acc = mega_dispatch<T>(p.kind, a, tile, smem_raw);
                if (a.red.kind != RED_NONE) {
                    __syncthreads();  // smem is reused as reduction scratch
                    grid_reduce_finish(acc, reinterpret_cast<double*>(smem_raw), a.red,
                                       (unsigned)p.ntiles, (unsigned)tile);
                }
                __syncthreads();  // the next tile reuses shared memory
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            // all threads' writes of this item (ordered by the barrier) and a
            // finished reduction, before its count
            __threadfence();
            atomicAdd(m.done + pi, 1);
        }
    }
}

}  // namespace

int mega_kind(int prec, int n, int axis) {
    (void)prec;
    for (int k = 0; k < kMegaPlanCount; ++k)
        if (kMegaPlans[k].n == n) return 2 * k + (axis > 0 ? 1 : 0);
    return -1;
}

int mega_threads_per_line(int kind) { return kMegaPlans[kind >> 1].p; }

int mega_plan_ls(int prec, int kind) {
    const MegaPlan& m = kMegaPlans[kind >> 1];
    const PassKernel* ks[8];
    const int nk = find_pass_kernels(prec, m.n, ks, 8);
    for (int i = 0; i < nk; ++i)
        if (ks[i]->ra == m.ra && ks[i]->rb == m.rb && ks[i]->rc == m.rc && ks[i]->p == m.p)
            return ks[i]->ls;
    return -1;
}

void* mega_kernel(int prec) {
    return prec == PREC_F32 ? (void*)&k_batch_mega<float> : (void*)&k_batch_mega<double>;
}

}  // namespace gpue
