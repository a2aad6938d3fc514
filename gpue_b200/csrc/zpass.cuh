// zpass.cuh -- the complex64 z pass (F K I along z) of a 3D field with its
// tiles brought in by TMA.
//
// A tile is CX = 16 adjacent x-columns of one y-row over all nz planes (the
// 16 z-lines of a 128-byte row segment).  One cp.async.bulk.tensor load per
// tile (a 3D tensor map over the field: box 16 x 1 x nz, complex64 moved as
// 8-byte elements) lands it in shared memory, completing on an mbarrier; the
// landing area is double-buffered, so the next tile's load is in flight while
// this one is transformed.  Threads (line c, thread t of P) read their values
// from the landing tile, run the forward transform, the kinetic factor and the
// inverse transform (exchanges through a separate scratch at a stride of 1
// mod 16 elements, so the 16 lines a half-warp touches fall on distinct
// banks), and store straight to HBM (16 adjacent columns per half-warp).  The
// arithmetic is that of the line pass's complex64 ops (pass.cuh).  The tensor
// map covers this GPU's own field only and no load uses cluster multicast.
// The mbarrier waits are bounded; a wait that gives up sets *err.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "plane.cuh"

namespace gpue {

template <typename T, int N, int RA, int RB, int P, int RC>
struct ZShape {
    using L = LineFFT<T, N, RA, RB, P, RC>;
    static constexpr int E = L::E;
    static constexpr int CX = 16;  // x-adjacent lines per tile
    static constexpr int THREADS = CX * P;
    static constexpr size_t TILE = (size_t)N * CX * sizeof(cx<T>);
    static constexpr int LSZ = ((smem_phys(N - 1) + 1 + 15) / 16) * 16 + 1;
    static constexpr size_t XCH = (size_t)CX * LSZ * sizeof(cx<T>);
    static constexpr size_t TWB = (size_t)N * 16;
    static constexpr size_t DB = (size_t)N * sizeof(float2);
    // + the two mbarriers, + 128 bytes to align the base for the TMA tiles
    static constexpr size_t SMEM = 2 * TILE + XCH + TWB + DB + 16 + 128;
    static_assert(std::is_same<T, float>::value, "complex64 z pass");
    static_assert(N <= 256, "a TMA box dimension holds at most 256 elements");
    static_assert(TILE % 128 == 0 && XCH % 16 == 0, "aligned regions");
    static_assert(L::kStageTableLen <= N, "the per-stage twiddle table fits its region");
};

// ops: F (z), K (separable, FP64-formed factor minus 1, scaled by 1/N and
// the optional norm-guard factor), I; in place on the field the tensor map
// covers (a.in == a.out).
template <typename T, int N, int RA, int RB, int P, int RC>
__global__ void __launch_bounds__(ZShape<T, N, RA, RB, P, RC>::THREADS, 2)
    k_zpass(const __grid_constant__ CUtensorMap tm, const PassArgs a) {
    using Z = ZShape<T, N, RA, RB, P, RC>;
    using L = typename Z::L;
    constexpr int E = Z::E;
    constexpr int CX = Z::CX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // TMA tile destinations are 128-byte aligned: align the base here (the
    // dynamic region follows any static shared variables)
    unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
    cx<T>* land = reinterpret_cast<cx<T>*>(smem);  // [2][N][CX]
    cx<T>* xch = reinterpret_cast<cx<T>*>(smem + 2 * Z::TILE);
    float4* tws = reinterpret_cast<float4*>(smem + 2 * Z::TILE + Z::XCH);
    float2* dz_s = reinterpret_cast<float2*>(smem + 2 * Z::TILE + Z::XCH + Z::TWB);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * Z::TILE + Z::XCH + Z::TWB + Z::DB);

    const int tid = threadIdx.x;
    L::build_stage_table(tws, reinterpret_cast<const float4*>(a.tw), tid, Z::THREADS);
    for (int i = tid; i < N; i += Z::THREADS) dz_s[i] = a.kd[2][i];
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    __syncthreads();
    const cx<T>* twp = reinterpret_cast<const cx<T>*>(tws);
    pdl_wait();

    const int ntx = a.nx / CX;
    const long ntiles = (long)ntx * a.ny;
    const long plane = (long)a.nx * a.ny;
    cx<T>* __restrict__ out = reinterpret_cast<cx<T>*>(a.out);
    const int c = tid % CX, t = tid / CX;
    const double ks = a.kscale_in ? a.kscale * *a.kscale_in : a.kscale;
    auto issue = [&](long tile, int b) {
        // order earlier generic-proxy reads of this buffer before the copy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const int x0 = (int)(tile % ntx) * CX, y = (int)(tile / ntx);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     ::"r"(smem_addr(bar + b)), "r"((unsigned)Z::TILE) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(land + (size_t)b * N * CX)),
            "l"(reinterpret_cast<uint64_t>(&tm)), "r"(x0), "r"(y), "r"(0),
            "r"(smem_addr(bar + b))
            : "memory");
    };

    bool ok = true;
    unsigned par[2] = {0u, 0u};
    int b = 0;
    long tile = blockIdx.x;
    if (tid == 0 && tile < ntiles) issue(tile, 0);
    for (; tile < ntiles; tile += gridDim.x, b ^= 1) {
        // every thread has read the other buffer (last iteration's tile)
        if (tid == 0 && tile + gridDim.x < ntiles) issue(tile + gridDim.x, b ^ 1);
        ok &= mbar_wait(bar + b, par[b], kPlaneWaitPolls);
        par[b] ^= 1u;
        const cx<T>* src = land + (size_t)b * N * CX;
        cx<T> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = src[L::index(t, e) * CX + c];
        __syncthreads();  // the tile is in registers: its buffer may take the next load
        const int x = (int)(tile % ntx) * CX + c, y = (int)(tile / ntx);
        cx<T>* sl = xch + c * Z::LSZ;
        auto sync = [] { __syncthreads(); };
        L::template forward<true>(v, t, sl, twp, sync);
        const cx<double> lf = cmul(ld2(a.kfac[0], x), ld2(a.kfac[1], y));
        op_kphase_f32<L>(v, t, dz_s, line_delta(lf), (float)ks);
#pragma unroll
        for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
        L::template forward<true>(v, t, sl, twp, sync);
#pragma unroll
        for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
        cx<T>* o = out + (long)y * a.nx + x;
#pragma unroll
        for (int e = 0; e < E; ++e) o[(long)L::index(t, e) * plane] = v[e];
    }
    if (!ok && a.err) atomicExch(a.err, 1);
    pdl_launch_dependents();
}

}  // namespace gpue
