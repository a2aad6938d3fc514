// tstream.cuh -- the complex64 pass kernels of the 3D step that move whole
// tiles with TMA: the XY pass (both in-plane transforms, x then y, in one
// launch) and the z pass (F K I along z).
//
// A tile is 16 lines of one kind:
//   x-tile  16 consecutive rows of one z-plane (a contiguous 16 x nx block)
//   y-tile  16 adjacent x-columns of one z-plane over all y
//   z-tile  16 adjacent x-columns of one y-row over all z
// It comes in by one cp.async.bulk.tensor load (this GPU's field, no
// multicast) and goes back, in place, by one bulk tensor store.  y- and
// z-tiles land with the 128-byte swizzle: their rows are 16 complex64 values
// (128 bytes), and the swizzle spreads a column over all banks, so the P
// threads of a line read (and write) their column without conflicts.  Every
// line's P threads sit in one warp, so the transform's exchanges need only
// __syncwarp: no compute warp waits for another.
//
// Roles: one producer warp (one active lane) and 16 * P / 32 compute warps.
// The producer takes tickets from a grid-wide counter, issues the loads into
// two landing buffers (full[b], mbarrier with a byte count), waits until the
// compute warps have written the tile back into its buffer (done[b]), issues
// the store, and once the buffer has been read out takes the next ticket for
// it.  The compute warps only wait for full[b].
//
// XY ordering.  Tickets follow: the x-tiles of plane g, then the y-tiles of
// plane g - LAG, for g = 0, 1, ...  A y-tile of plane z may load only after
// all x-tiles of plane z are stored (a per-plane count, raised with release
// semantics by each x-tile's producer once its store is complete, and read
// with acquire semantics); by then the plane is normally still in L2, so the
// field crosses HBM once in and once out.  The producer counts an x-tile as
// soon as its store completes, after it has refilled the buffer (the compute
// warps are busy with the other buffer meanwhile).  LAG (64 planes by
// default: shorter lags leave y-tiles waiting, longer ones overflow L2) is
// set per context.  A producer whose next y-tile's plane is not ready only
// marks the buffer pending, and waits (bounded) for it when that buffer's
// turn comes, when every tile it held with a smaller ticket is stored and
// counted.  A waited-for x-tile therefore always has a smaller ticket
// than the wait, and a CTA holding one either is not waiting or waits for a
// still smaller ticket: no cycle, and the smallest waiting ticket's x-tiles
// are all held by CTAs that finish them.  Every wait is bounded; one that
// gives up sets *err (the host reports GPUE_ERR_TIMEOUT), and the kernel then
// drains its copies in flight before it returns.
//
// The counters reset themselves: the last CTA to finish clears the ticket,
// the per-plane counts and its own finish count, so consecutive launches need
// no memset between them.
//
// Ops.  XY forward: x-tiles [scale] V/2 Fx, y-tiles Fy.  XY inverse: x-tiles
// Ix, y-tiles Iy V/2 [norm].  z pass: Fz K Iz.  The arithmetic is that of the
// line pass's complex64 ops (pass.cuh), with the per-stage twiddle table and
// the factor tables in shared memory.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include <type_traits>

#include "plane.cuh"

namespace gpue {

enum : int { TS_XY_FWD = 0, TS_XY_INV = 1, TS_Z = 2 };
enum : int { TILE_X = 0, TILE_Y = 1, TILE_Z = 2, TILE_END = -1 };

template <typename T, int N, int RA, int RB, int P, int RC>
struct TSShape {
    using L = LineFFT<T, N, RA, RB, P, RC>;
    static constexpr int E = L::E;
    static constexpr int LT = 16;           // lines per tile
    static constexpr int CT = LT * P;       // compute threads
    static constexpr int CW = CT / 32;      // compute warps
    static constexpr int THREADS = CT + 32; // + the producer warp
    static constexpr size_t TILE = (size_t)N * LT * sizeof(cx<T>);
    static constexpr int LS = L::LS;
    static constexpr size_t XCH = (size_t)LT * LS * sizeof(cx<T>);
    static constexpr size_t TWB = (size_t)N * 16;
    static constexpr size_t DB = (size_t)N * sizeof(float2);
    static constexpr size_t OFF_XCH = 2 * TILE;
    static constexpr size_t OFF_TW = OFF_XCH + XCH;
    static constexpr size_t OFF_D = OFF_TW + TWB;
    static constexpr size_t OFF_BAR = OFF_D + 2 * DB;
    // + 4 mbarriers, 2 tile slots and a 256-plane ready bitmap, + 1024 bytes
    // to align the base (the 128-byte swizzle repeats every 1024 bytes of the
    // destination address)
    static constexpr size_t SMEM = OFF_BAR + 96 + 1024;
    static_assert(std::is_same<T, float>::value, "complex64 tile stream");
    static_assert(N <= 256 && N % LT == 0, "a TMA box dimension holds at most 256 elements");
    static_assert(CT % 32 == 0 && 32 % P == 0, "whole warps; a line's threads in one warp");
    static_assert(TILE % 1024 == 0, "landing tiles keep the swizzle alignment");
    static_assert(OFF_TW % 16 == 0 && OFF_BAR % 16 == 0, "aligned regions");
    static_assert(L::kStageTableLen <= N, "the per-stage twiddle table fits its region");
};

// Element (row r, column c) of a [rows][16] complex64 tile landed with the
// 128-byte swizzle: the 16-byte chunk index (c / 2) is XORed with r mod 8.
__device__ __forceinline__ int sw128(int r, int c) {
    return r * 16 + ((((c >> 1) ^ (r & 7)) << 1) | (c & 1));
}

// XY ticket t -> (kind, plane, tile): xi x-tiles and yi y-tiles per plane
// (32-bit arithmetic: a launch has nz * (xi + yi) < 2^31 tiles).
__device__ __forceinline__ int xy_ticket(unsigned t, unsigned xi, unsigned yi, unsigned nz,
                                         unsigned lag, int& z, int& tile) {
    const unsigned t1 = lag * xi, t2 = t1 + (nz - lag) * (xi + yi);
    if (t < t1) {
        z = (int)(t / xi);
        tile = (int)(t % xi);
        return TILE_X;
    }
    if (t < t2) {
        const unsigned u = t - t1;
        const int w = (int)(u % (xi + yi));
        const int g = (int)(lag + u / (xi + yi));
        if (w < xi) {
            z = g;
            tile = w;
            return TILE_X;
        }
        z = g - lag;
        tile = w - xi;
        return TILE_Y;
    }
    const unsigned u = t - t2;
    z = (int)(nz - lag + u / yi);
    tile = (int)(u % yi);
    return TILE_Y;
}

// The x-tile count of a plane, read with acquire semantics (the stores it
// counts happen before what follows), and raised with release semantics.
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(int* p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Nanoseconds of the GPU's global timer: the bound of the plane wait.
__device__ __forceinline__ uint64_t gpu_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
constexpr uint64_t kPlaneWaitNs = 1000000000ull;  // a y-tile waits at most 1 s for its plane

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}

// One bounded poll of phase `parity` of an mbarrier (true: it has completed).
__device__ __forceinline__ bool mbar_test(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2; "
        "selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

template <typename T, int N, int RA, int RB, int P, int RC, int KIND>
__global__ void __launch_bounds__(TSShape<T, N, RA, RB, P, RC>::THREADS, 2)
    k_tstream(const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
              const PassArgs a, const XYCounters k) {
    using S_ = TSShape<T, N, RA, RB, P, RC>;
    using L = typename S_::L;
    constexpr int E = S_::E;
    constexpr int LT = S_::LT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
    cx<T>* land = reinterpret_cast<cx<T>*>(smem);  // [2] tiles
    cx<T>* xch = reinterpret_cast<cx<T>*>(smem + S_::OFF_XCH);
    float4* tws = reinterpret_cast<float4*>(smem + S_::OFF_TW);
    // factor tables: V/2 along x and y (XY), or the K factor along z as
    // (d.x, d.y, d.y, d.x) for the packed product (z pass)
    float2* d0_s = reinterpret_cast<float2*>(smem + S_::OFF_D);
    float2* d1_s = d0_s + N;
    float4* dz_s = reinterpret_cast<float4*>(smem + S_::OFF_D);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S_::OFF_BAR);
    uint64_t* done = full + 2;
    int4* slot = reinterpret_cast<int4*>(smem + S_::OFF_BAR + 32);  // [2] (kind, z, tile)
    unsigned* s_ready = reinterpret_cast<unsigned*>(smem + S_::OFF_BAR + 64);  // planes ready

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    L::build_stage_table(tws, reinterpret_cast<const float4*>(a.tw), tid, S_::THREADS);
    for (int i = tid; i < N; i += S_::THREADS) {
        if constexpr (KIND == TS_Z) {
            const float2 d = a.kd[2][i];
            dz_s[i] = make_float4(d.x, d.y, d.y, d.x);
        } else {
            d0_s[i] = a.vd[0][i];
            d1_s[i] = a.vd[1][i];
        }
    }
    if (tid == 0) {
        mbar_init(full, 1);
        mbar_init(full + 1, 1);
        mbar_init(done, S_::CW);
        mbar_init(done + 1, S_::CW);
    }
    __syncthreads();
    pdl_wait();  // the field and the scale are the previous kernel's output
    // a converged solve of a batched run (its active flag cleared by the
    // previous check) is left as it is: every CTA returns before touching the
    // field or the work counters
    if (a.active && *reinterpret_cast<const volatile int*>(a.active) == 0) {
        pdl_launch_dependents();
        return;
    }

    const int nz = a.nz;
    const int xi = a.ny / LT, yi = a.nx / LT;  // x-tiles (and y- or z-tiles) per plane
    bool ok = true;
    KSum acc{0.0, 0.0};

    if (warp == S_::CW) {
        // ------------------------------------------------------ producer
        if (lane == 0) {
            const int lag = k.lag < 1 ? 1 : k.lag < nz ? k.lag : nz;
            const int need = xi + k.wait_extra;  // x-tiles a plane's y-tiles wait for
            const long total = KIND == TS_Z ? (long)yi * a.ny : (long)nz * (xi + yi);
            // per landing buffer: its ticket and tile, whether its load waits
            // for a plane, the parity of its next done phase, the phases begun
            // on its full barrier
            struct Buf {
                long tk;
                int kind, z, tile;
                bool pend;
                unsigned dpar, nfull;
            };
            Buf B0{0, 0, 0, 0, false, 0u, 0u}, B1{0, 0, 0, 0, false, 0u, 0u};
            for (int i = 0; i < 8; ++i) s_ready[i] = 0u;
            auto known_ready = [&](int z) {
                return z < 256 && ((s_ready[z >> 5] >> (z & 31)) & 1u);
            };
            auto see_ready = [&](int z) {
                // (after an acquire read of the count) the other CTAs' stores
                // of this plane before TMA reads of it
                asm volatile("fence.proxy.async.global;" ::: "memory");
                if (z < 256) s_ready[z >> 5] |= 1u << (z & 31);
            };
            auto count = [&](int z) {
                // the store is complete: publish it to the y-tiles of plane z
                asm volatile("fence.proxy.async.global;" ::: "memory");
                red_release_add(k.done_x + z, 1);
            };
            auto map_of = [&](int kd) -> uint64_t {
                return reinterpret_cast<uint64_t>(kd == TILE_Y ? &tm1 : &tm0);
            };
            auto coords = [&](const Buf& m, int& c0, int& c1, int& c2) {
                if (m.kind == TILE_X) {
                    c0 = 0, c1 = m.tile * LT, c2 = m.z;
                } else if (m.kind == TILE_Y) {
                    c0 = m.tile * LT, c1 = 0, c2 = m.z;
                } else {
                    c0 = m.tile * LT, c1 = m.z, c2 = 0;  // z-tile: z holds the y-row
                }
            };
            auto load = [&](auto bc, Buf& m) {
                constexpr int b = decltype(bc)::value;
                int c0, c1, c2;
                coords(m, c0, c1, c2);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                             ::"r"(smem_addr(full + b)), "r"((unsigned)S_::TILE) : "memory");
                asm volatile(
                    "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
                    "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(land + (size_t)b * N * LT)),
                    "l"(map_of(m.kind)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(full + b))
                    : "memory");
                m.nfull++;
            };
            // buffer b takes ticket m.tk: load now, mark pending, or end
            auto prepare = [&](auto bc, Buf& m) {
                constexpr int b = decltype(bc)::value;
                m.pend = false;
                if (m.tk >= total) {
                    slot[b] = make_int4(TILE_END, 0, 0, 0);
                    mbar_arrive(full + b);
                    m.nfull++;
                    return;
                }
                if constexpr (KIND == TS_Z) {
                    m.kind = TILE_Z;
                    m.z = (int)((unsigned)m.tk / (unsigned)yi);
                    m.tile = (int)((unsigned)m.tk % (unsigned)yi);
                } else {
                    m.kind = xy_ticket((unsigned)m.tk, xi, yi, nz, lag, m.z, m.tile);
                }
                slot[b] = make_int4(m.kind, m.z, m.tile, 0);
                if (m.kind == TILE_Y && !known_ready(m.z)) {
                    if (ld_acquire(k.done_x + m.z) < need) {
                        m.pend = true;
                        return;
                    }
                    see_ready(m.z);
                }
                load(bc, m);
            };
            unsigned long long nxt = 0;
            // one turn of buffer b: false when the stream has ended
            auto turn = [&](auto bc, Buf& m) -> bool {
                constexpr int b = decltype(bc)::value;
                if (m.tk >= total) return false;  // so is the other buffer's (a later ticket)
                if (m.pend) {
                    // every tile held with a smaller ticket is stored and
                    // counted (x-tiles are counted as their store completes)
                    const uint64_t t0 = gpu_ns();
                    while (ld_acquire(k.done_x + m.z) < need) {
                        if (gpu_ns() - t0 > kPlaneWaitNs) {
                            ok = false;
                            break;
                        }
                        __nanosleep(64);
                    }
                    see_ready(m.z);
                    load(bc, m);
                    m.pend = false;
                }
                if (!mbar_wait(done + b, m.dpar, kPlaneWaitPolls)) {
                    ok = false;
                    return false;
                }
                m.dpar ^= 1u;
                int c0, c1, c2;
                coords(m, c0, c1, c2);
                asm volatile(
                    "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group "
                    "[%0, {%1, %2, %3}], [%4];" ::"l"(map_of(m.kind)),
                    "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(land + (size_t)b * N * LT))
                    : "memory");
                asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                const int stored_x = m.kind == TILE_X ? m.z : -1;
                // refill the buffer first: the compute warps wait for it
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                m.tk = (long)nxt;
                prepare(bc, m);
                if (m.tk < total) nxt = atomicAdd(k.ticket, 1ull);
                if (stored_x >= 0) {
                    // the compute warps have the other buffer's tile: wait for
                    // this store to complete and count it now
                    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
                    count(stored_x);
                }
                return true;
            };
            using I0 = std::integral_constant<int, 0>;
            using I1 = std::integral_constant<int, 1>;
            B0.tk = (long)atomicAdd(k.ticket, 1ull);
            prepare(I0{}, B0);
            B1.tk = (long)atomicAdd(k.ticket, 1ull);
            prepare(I1{}, B1);
            nxt = atomicAdd(k.ticket, 1ull);
            while (turn(I0{}, B0) && turn(I1{}, B1)) {
            }
            asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
            if (!ok) {
                // a wait gave up: let the loads still in flight land before
                // the shared memory is released
                for (unsigned p = 0; B0.nfull && p < kPlaneWaitPolls; ++p)
                    if (mbar_test(full, (B0.nfull - 1) & 1u)) break;
                for (unsigned p = 0; B1.nfull && p < kPlaneWaitPolls; ++p)
                    if (mbar_test(full + 1, (B1.nfull - 1) & 1u)) break;
            }
            // the last CTA to finish clears the counters for the next launch
            __threadfence();
            if (atomicAdd(k.finish, 1u) == gridDim.x - 1) {
                *k.ticket = 0ull;
                for (int z = 0; z < nz; ++z) k.done_x[z] = 0;
                __threadfence();
                *k.finish = 0u;
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------- compute warps
        const int l = tid / P, t = tid % P;
        const cx<T>* twp = reinterpret_cast<const cx<T>*>(tws);
        cx<T>* sl = xch + l * S_::LS;
        auto sync = [] { __syncwarp(); };
        const double sc = (KIND == TS_XY_FWD && a.ops[0]) ? *a.scale_in : 1.0;
        const double ks = KIND == TS_Z ? (a.kscale_in ? a.kscale * *a.kscale_in : a.kscale)
                                       : 0.0;
        unsigned fpar = 0u;  // bit b: parity of buffer b's next full phase
        int b = 0;
        for (;;) {
            if (!mbar_wait(full + b, (fpar >> b) & 1u, kPlaneWaitPolls)) {
                ok = false;
                break;
            }
            fpar ^= 1u << b;
            const int4 inf = slot[b];
            if (inf.x == TILE_END) break;
            const int z = inf.y, tile = inf.z;
            cx<T>* tb = land + (size_t)b * N * LT;
            const bool rows = inf.x == TILE_X;
            cx<T> v[E];
            if (rows) {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e] = tb[l * N + L::index(t, e)];
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e] = tb[sw128(L::index(t, e), l)];
            }
            if constexpr (KIND == TS_XY_FWD) {
                if (rows) {
                    const int y = tile * LT + l;
                    const cx<double> lf =
                        cscale(cmul(ld2(a.vfac[1], y), ld2(a.vfac[2], z)), sc);
                    // the pending scale is folded into the factor, so the
                    // density of the unscaled values takes it squared
                    op_vhalf_f32<L>(v, t, d0_s, line_delta(lf), a, a.nl_coef * sc * sc);
                }
                L::template forward<true>(v, t, sl, twp, sync);
            } else if constexpr (KIND == TS_XY_INV) {
                L::template forward<true, true>(v, t, sl, twp, sync);  // inverse
                if (!rows) {
                    const int x = tile * LT + l;
                    const cx<double> lf = cmul(ld2(a.vfac[0], x), ld2(a.vfac[2], z));
                    op_vhalf_f32<L>(v, t, d1_s, line_delta(lf), a, a.nl_coef);
                    if (a.red.kind == RED_NORM) op_norm_f32<E>(v, acc);
                }
            } else {
                const int x = tile * LT + l;  // z holds the y-row
                L::template forward<true>(v, t, sl, twp, sync);
                const cx<double> lf = cmul(ld2(a.kfac[0], x), ld2(a.kfac[1], z));
                op_kphase_f32_packed<L>(v, t, dz_s, line_delta(lf), (float)ks);
                L::template forward<true, true>(v, t, sl, twp, sync);  // inverse
            }
            if (rows) {
#pragma unroll
                for (int e = 0; e < E; ++e) tb[l * N + L::index(t, e)] = v[e];
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) tb[sw128(L::index(t, e), l)] = v[e];
            }
            // this thread's writes before the bulk store reads the buffer
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(done + b);
            b ^= 1;
        }
    }
    if (!ok && a.err) atomicExch(a.err, 1);
    pdl_launch_dependents();
    if (KIND == TS_XY_INV && a.red.kind != RED_NONE) {
        __syncthreads();
        grid_reduce_finish(acc, reinterpret_cast<double*>(xch), a.red, gridDim.x, blockIdx.x);
    }
}

}  // namespace gpue
