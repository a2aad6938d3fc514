// xystream.cuh -- both in-plane transforms of a 3D field (x then y) in one
// pass, without thread-block clusters: the field's x-tiles and y-tiles are
// independent work items, ordered so a plane's y-tiles run after its x-tiles
// while the x output is still in L2.
//
// Work is done in tiles of 16 lines: an x-tile is 16 consecutive rows of one
// z-plane (a contiguous 16 x nx block), a y-tile 16 adjacent x-columns of one
// z-plane over all y.  Tickets, taken with an atomic counter by resident CTAs,
// follow the order: the x-tiles of plane g, then the y-tiles of plane g - LAG,
// for g = 0, 1, ...  A y-tile of plane z waits (bounded) until all x-tiles of
// plane z are done (a per-plane count), and by then the x output it reads is
// normally still in L2, so the field crosses HBM once in and once out.  A
// tile comes in by one TMA load (cp.async.bulk.tensor, this GPU's field, no
// multicast) into a double-buffered landing area: the next ticket's load is
// issued while the current tile is transformed.  Tiles are transformed in
// registers with exchanges through shared memory (per-stage twiddle tables,
// the V/2 factor tables and the complex64 phase ops of pass.cuh) and stored
// straight back in place.  Forward: x-tiles [scale] V/2 Fx, y-tiles Fy.
// Inverse: x-tiles Ix, y-tiles Iy V/2 [norm].
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "plane.cuh"

namespace gpue {

constexpr int kXYLag = 32;  // planes between a plane's x-tiles and its y-tiles

template <typename T, int N, int RA, int RB, int P, int RC>
struct XYShape {
    using L = LineFFT<T, N, RA, RB, P, RC>;
    static constexpr int E = L::E;
    static constexpr int LT = 16;  // lines per tile
    static constexpr int THREADS = LT * P;
    static constexpr size_t TILE = (size_t)N * LT * sizeof(cx<T>);
    static constexpr int LSR = L::LS;
    static constexpr int LSC = ((smem_phys(N - 1) + 1 + 15) / 16) * 16 + 1;
    static constexpr int SLS = LSR > LSC ? LSR : LSC;
    static constexpr size_t XCH = (size_t)LT * SLS * sizeof(cx<T>);
    static constexpr size_t TWB = (size_t)N * 16;
    static constexpr size_t DB = (size_t)N * sizeof(float2);
    // + the two mbarriers, + 128 bytes to align the base for the TMA tiles
    static constexpr size_t SMEM = 2 * TILE + XCH + TWB + 2 * DB + 16 + 128;
    static_assert(std::is_same<T, float>::value, "complex64 xy pass");
    static_assert(N <= 256 && N % LT == 0, "a TMA box dimension holds at most 256 elements");
    static_assert(P <= 32 && 32 % P == 0, "a row's threads sit in one warp");
    static_assert(TILE % 128 == 0 && XCH % 16 == 0, "aligned regions");
    static_assert(L::kStageTableLen <= N, "the per-stage twiddle table fits its region");
};

// Ticket t -> (is_y, plane, tile): xi x-tiles and yi y-tiles per plane.
__device__ __forceinline__ bool xy_item(long t, int xi, int yi, int nz, int lag, int& z,
                                        int& tile) {
    const long t1 = (long)lag * xi, t2 = t1 + (long)(nz - lag) * (xi + yi);
    if (t < t1) {
        z = (int)(t / xi);
        tile = (int)(t % xi);
        return false;
    }
    if (t < t2) {
        const long u = t - t1;
        const int w = (int)(u % (xi + yi));
        const int g = lag + (int)(u / (xi + yi));
        if (w < xi) {
            z = g;
            tile = w;
            return false;
        }
        z = g - lag;
        tile = w - xi;
        return true;
    }
    const long u = t - t2;
    z = nz - lag + (int)(u / yi);
    tile = (int)(u % yi);
    return true;
}

template <typename T, int N, int RA, int RB, int P, int RC, bool INV>
__global__ void __launch_bounds__(XYShape<T, N, RA, RB, P, RC>::THREADS, 2)
    k_xy(const __grid_constant__ CUtensorMap tmx, const __grid_constant__ CUtensorMap tmy,
         const PassArgs a, const XYCounters k) {
    using S_ = XYShape<T, N, RA, RB, P, RC>;
    using L = typename S_::L;
    constexpr int E = S_::E;
    constexpr int LT = S_::LT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // TMA tile destinations are 128-byte aligned: static shared variables (the
    // ticket slots, the reduction's flag) come first, so align the base here
    unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
    cx<T>* land = reinterpret_cast<cx<T>*>(smem);  // [2][LT][N] or [2][N][LT]
    cx<T>* xch = reinterpret_cast<cx<T>*>(smem + 2 * S_::TILE);
    float4* tws = reinterpret_cast<float4*>(smem + 2 * S_::TILE + S_::XCH);
    float2* dx_s = reinterpret_cast<float2*>(smem + 2 * S_::TILE + S_::XCH + S_::TWB);
    float2* dy_s = dx_s + N;
    uint64_t* bar =
        reinterpret_cast<uint64_t*>(smem + 2 * S_::TILE + S_::XCH + S_::TWB + 2 * S_::DB);
    __shared__ long s_ticket[2];

    const int tid = threadIdx.x;
    L::build_stage_table(tws, reinterpret_cast<const float4*>(a.tw), tid, S_::THREADS);
    for (int i = tid; i < N; i += S_::THREADS) {
        dx_s[i] = a.vd[0][i];
        dy_s[i] = a.vd[1][i];
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
    }
    __syncthreads();
    const cx<T>* twp = reinterpret_cast<const cx<T>*>(tws);
    pdl_wait();

    const int nz = a.nz;
    const int xi = a.ny / LT, yi = a.nx / LT;  // x-tiles and y-tiles per plane
    const int lag = kXYLag < nz ? kXYLag : nz;
    const long total = (long)nz * (xi + yi);
    const long plane = (long)a.nx * a.ny;
    cx<T>* __restrict__ out = reinterpret_cast<cx<T>*>(a.out);
    bool ok = true;

    // Thread 0 keeps two tiles in flight, one per landing buffer.  A ticket is
    // taken one tile ahead of its load (the atomic's latency overlaps a
    // tile's arithmetic).  A y-tile whose plane is not known ready yet is only
    // marked pending, and its load is issued (after a bounded wait) when its
    // turn comes, so a CTA never waits while it holds a tile it has not
    // transformed: the x-tiles a wait needs are then all held by CTAs that
    // finish them without waiting.  Planes seen ready are remembered, so most
    // y-tiles neither read the counts nor fence.
    bool pending[2] = {false, false};
    unsigned ready[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // planes seen ready (the first 256)
    auto known_ready = [&](int z) {
        return z < 256 && ((ready[z >> 5] >> (z & 31)) & 1u);
    };
    auto issue = [&](int b, long t) {
        int z, tile;
        const bool is_y = xy_item(t, xi, yi, nz, lag, z, tile);
        if (is_y && !known_ready(z)) {
            const volatile int* d = k.done_x + z;
            unsigned polls = 0;
            while (*d < xi) {
                if (++polls >= kPlaneWaitPolls) {
                    ok = false;
                    break;
                }
                __nanosleep(32);
            }
            __threadfence();
            // the other CTAs' x-tile stores before TMA reads of this plane
            asm volatile("fence.proxy.async.global;" ::: "memory");
            if (z < 256) ready[z >> 5] |= 1u << (z & 31);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     ::"r"(smem_addr(bar + b)), "r"((unsigned)S_::TILE) : "memory");
        const unsigned dst = smem_addr(land + (size_t)b * N * LT);
        if (is_y)
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
                "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                "l"(reinterpret_cast<uint64_t>(&tmy)), "r"(tile * LT), "r"(0), "r"(z),
                "r"(smem_addr(bar + b))
                : "memory");
        else
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
                "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
                "l"(reinterpret_cast<uint64_t>(&tmx)), "r"(0), "r"(tile * LT), "r"(z),
                "r"(smem_addr(bar + b))
                : "memory");
    };
    // buffer b takes ticket t: load now, or mark pending
    auto assign = [&](int b, long t) {
        s_ticket[b] = t;
        pending[b] = false;
        if (t >= total) return;
        int z, tile;
        if (xy_item(t, xi, yi, nz, lag, z, tile) && !known_ready(z) &&
            *reinterpret_cast<const volatile int*>(k.done_x + z) < xi) {
            pending[b] = true;
            return;
        }
        issue(b, t);
    };

    const double sc = (!INV && a.ops[0]) ? *a.scale_in : 1.0;
    KSum acc{0.0, 0.0};
    unsigned par[2] = {0u, 0u};
    int b = 0;
    if (tid == 0) {
        assign(0, (long)atomicAdd(k.ticket, 1ull));
        assign(1, (long)atomicAdd(k.ticket, 1ull));
    }
    __syncthreads();
    for (;;) {
        const long t = s_ticket[b];
        if (t >= total) break;
        unsigned long long t_next = 0;
        if (tid == 0) {
            if (pending[b]) issue(b, t);  // its plane is ready by now, or soon
            t_next = atomicAdd(k.ticket, 1ull);  // for this buffer's next tile
        }
        ok &= mbar_wait(bar + b, par[b], kPlaneWaitPolls);
        par[b] ^= 1u;
        int z, tile;
        const bool is_y = xy_item(t, xi, yi, nz, lag, z, tile);
        const cx<T>* src = land + (size_t)b * N * LT;
        cx<T> v[E];
        if (!is_y) {
            // x-tile: rows tile*16 .. +15 of plane z; thread rt of row rl
            const int rt = tid % P, rl = tid / P;
            const int y = tile * LT + rl;
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = src[rl * N + L::index(rt, e)];
            cx<T>* sl = xch + rl * S_::SLS;
            auto sync = [] { __syncwarp(); };
            if constexpr (!INV) {
                const cx<double> lf = cscale(cmul(ld2(a.vfac[1], y), ld2(a.vfac[2], z)), sc);
                // the pending scale is folded into the factor, so the density
                // of the unscaled values takes it squared
                op_vhalf_f32<L>(v, rt, dx_s, line_delta(lf), a, a.nl_coef * sc * sc);
                L::template forward<true>(v, rt, sl, twp, sync);
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
                L::template forward<true>(v, rt, sl, twp, sync);
#pragma unroll
                for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
            }
            cx<T>* o = out + (long)z * plane + (long)y * a.nx;
#pragma unroll
            for (int e = 0; e < E; ++e) o[L::index(rt, e)] = v[e];
        } else {
            // y-tile: x-columns tile*16 .. +15 of plane z; thread ct of column cc
            const int cc = tid % LT, ct = tid / LT;
            const int x = tile * LT + cc;
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = src[L::index(ct, e) * LT + cc];
            cx<T>* sl = xch + cc * S_::LSC;
            auto sync = [] { __syncthreads(); };
            if constexpr (!INV) {
                L::template forward<true>(v, ct, sl, twp, sync);
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
                L::template forward<true>(v, ct, sl, twp, sync);
#pragma unroll
                for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
                const cx<double> lf = cmul(ld2(a.vfac[0], x), ld2(a.vfac[2], z));
                op_vhalf_f32<L>(v, ct, dy_s, line_delta(lf), a, a.nl_coef);
                if (a.red.kind == RED_NORM) op_norm_f32<E>(v, acc);
            }
            cx<T>* o = out + (long)z * plane + x;
#pragma unroll
            for (int e = 0; e < E; ++e) o[(long)L::index(ct, e) * a.nx] = v[e];
        }
        // every thread's stores issued, buffer b and the exchange scratch free
        __syncthreads();
        if (tid == 0) {
            if (!is_y) {
                // this x-tile's rows (all threads', ordered by the barrier)
                // before its plane's count
                __threadfence();
                atomicAdd(k.done_x + z, 1);
            }
            assign(b, (long)t_next);
        }
        b ^= 1;
    }
    if (!ok && a.err) atomicExch(a.err, 1);
    pdl_launch_dependents();
    if (INV && a.red.kind != RED_NONE) {
        __syncthreads();
        grid_reduce_finish(acc, reinterpret_cast<double*>(xch), a.red, gridDim.x, blockIdx.x);
    }
}

}  // namespace gpue
