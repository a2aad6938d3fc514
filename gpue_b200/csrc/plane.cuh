// plane.cuh -- one full-field pass that transforms both in-plane axes (x and
// y) of a 3D field, so a split step needs three full-field passes instead of
// five:  XY[scale V/2 Fx Fy] . Z[Fz K Iz] . XY[Ix Iy V/2 norm].
//
// A thread-block cluster owns one z-plane at a time (N x N points, N = nx =
// ny).  Its CS = N/32 CTAs each own 32 rows.  Per plane:
//   1. once the cluster has finished reading the previous plane, the CTA's
//      32 rows land in its exchange buffer X by one asynchronous bulk copy
//      per row (cp.async.bulk, completing on an mbarrier, one row per padded
//      row slot);
//   2. in two rounds of 16 rows the rows go through the row ops and the x
//      transform in registers (its exchanges through a scratch buffer S) and
//      back into their X slots in the padded layout;
//   3. after a cluster barrier every CTA reads its 32 columns out of all the
//      cluster's X buffers through distributed shared memory (two rounds of
//      16 columns), runs the y transform and the column ops, and stores the
//      columns to HBM (16 adjacent columns per half-warp: 128-byte segments).
// The 2D transform is separable, so the inverse pass also runs x first; its
// V/2 and norm come in the column phase.  Planes are walked persistently,
// cluster c taking planes c, c + #clusters, ...  A CTA needs ~112 KB of shared
// memory and 256 threads, so two CTAs (of different clusters) share an SM and
// one's barrier and load waits overlap the other's arithmetic.
//
// Shared memory per CTA: X (32 row slots at the line FFT's padded stride), S
// (16 lines; columns at a stride of 1 mod 16 elements so the 16 columns a
// half-warp touches fall on distinct banks), and copies of the twiddle table
// and the x and y V/2 factor tables.
//
// The transforms, phase factors, scalings and the deferred renormalisation are
// those of the complex64 line passes (pass.cuh); only the order in which the
// two in-plane transforms and their data movement happen differs.  Every wait
// is bounded: an mbarrier wait that gives up sets *err and the kernel carries
// on (keeping the cluster barriers in step) so the host sees a status, not a
// hang.

#pragma once

#include <stdint.h>

#include <type_traits>

#include "pass.cuh"

namespace gpue {

// ----------------------------------------------------- PTX for the cluster --

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_index() {
    unsigned r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_count() {
    unsigned r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// the shared::cluster address of `addr` (a shared::cta address) in CTA `rank`
__device__ __forceinline__ unsigned dsmem_map(unsigned addr, unsigned rank) {
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
template <typename T>
__device__ __forceinline__ cx<T> dsmem_load(unsigned addr) {
    cx<T> v;
    if constexpr (sizeof(T) == 4)
        asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];"
                     : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
    else
        asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];"
                     : "=d"(v.x), "=d"(v.y) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One bulk global -> shared copy of `bytes` (a multiple of 16, both addresses
// 16-byte aligned) that completes on mbarrier b; the calling thread also arms b.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          uint64_t* b) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(b))
        : "memory");
}
// Waits for phase `parity` of b to complete; false if it has not after
// `limit` polls (each poll may block the thread for a short while).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity, unsigned limit) {
    for (unsigned i = 0; i < limit; ++i) {
        unsigned ok;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
            "selp.u32 %0, 1, 0, p; }"
            : "=r"(ok)
            : "r"(smem_addr(b)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

constexpr unsigned kPlaneWaitPolls = 1u << 22;

// ------------------------------------------------------------ the kernel --

// LPR_ = 16: two rounds of 16 lines per phase, 16 P threads, two CTAs per SM
// (measured faster on the 256^3 ground state than one 32-line round of 32 P
// threads at one CTA per SM: 145 vs 185 us per pass)
template <typename T, int N, int RA, int RB, int P, int RC, int LPR_ = 16>
struct PlaneShape {
    using L = LineFFT<T, N, RA, RB, P, RC>;
    static constexpr int E = L::E;
    static constexpr int RPC = 32;         // rows (then columns) per CTA
    static constexpr int LPR = LPR_;       // lines transformed at once (a round)
    static constexpr int MINB = 512 / (LPR_ * P) > 1 ? 512 / (LPR_ * P) : 1;  // CTAs per SM
    static constexpr int CS = N / RPC;     // CTAs per cluster: one plane
    static constexpr int THREADS = LPR * P;
    static constexpr int LSR = L::LS;      // row stride of X (elements)
    static constexpr int LSC = ((smem_phys(N - 1) + 1 + 15) / 16) * 16 + 1;  // columns in S
    static constexpr int SLS = LSR > LSC ? LSR : LSC;  // line stride of S
    static constexpr size_t XB = (size_t)RPC * LSR * sizeof(cx<T>);
    static constexpr size_t SB = (size_t)LPR * SLS * sizeof(cx<T>);
    static constexpr size_t TWB = (size_t)N * 16;       // (hi, lo) float pairs
    static constexpr size_t DB = (size_t)N * sizeof(float2);  // one axis' factor - 1
    static constexpr size_t SMEM = XB + SB + TWB + 2 * DB + 16;  // + two mbarriers
    static_assert(std::is_same<T, float>::value, "complex64 plane passes");
    static_assert(N % RPC == 0 && CS >= 1 && CS <= 8, "plane of 32-row slices, <= 8 CTAs");
    static_assert(P <= 32 && 32 % P == 0, "a row's threads sit in one warp");
    static_assert(RPC % LPR == 0 && (LPR == 16 || LPR == 32), "whole rounds of lines");
    static_assert((LSR * sizeof(cx<T>)) % 16 == 0 && (N * sizeof(cx<T>)) % 16 == 0,
                  "row slots and rows are whole 16-byte units (bulk copies)");
    static_assert(XB % 16 == 0 && SB % 16 == 0, "16-byte regions");
};

// INV = false: rows [scale] V/2 Fx, columns Fy.
// INV = true:  rows Ix, columns Iy V/2 [norm].
// a.ops[0] != 0 asks for the deferred scale (forward pass only); a.red.kind
// RED_NORM for the norm (inverse pass only).
template <typename T, int N, int RA, int RB, int P, int RC, int LPR_, bool INV>
__global__ void __launch_bounds__(PlaneShape<T, N, RA, RB, P, RC, LPR_>::THREADS,
                                  PlaneShape<T, N, RA, RB, P, RC, LPR_>::MINB)
    k_plane(const PassArgs a) {
    using S_ = PlaneShape<T, N, RA, RB, P, RC, LPR_>;
    using L = typename S_::L;
    constexpr int E = S_::E;
    constexpr int RPC = S_::RPC;
    constexpr int LPR = S_::LPR;
    static_assert(L::kStageTableLen <= N, "the per-stage twiddle table fits its region");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* X = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* Sx = reinterpret_cast<cx<T>*>(smem_raw + S_::XB);
    float4* tws = reinterpret_cast<float4*>(smem_raw + S_::XB + S_::SB);
    float2* dx_s = reinterpret_cast<float2*>(smem_raw + S_::XB + S_::SB + S_::TWB);
    float2* dy_s = dx_s + N;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + S_::XB + S_::SB + S_::TWB + 2 * S_::DB);

    const int tid = threadIdx.x;
    const unsigned rank = cluster_rank();
    const long nz = a.nz;
    const long zstep = cluster_count();
    const size_t plane = (size_t)N * N;
    const cx<T>* __restrict__ in = reinterpret_cast<const cx<T>*>(a.in);
    cx<T>* __restrict__ out = reinterpret_cast<cx<T>*>(a.out);

    // the tables this pass reads per element, staged once (they do not depend
    // on the state, so before the wait on the previous kernel)
    L::build_stage_table(tws, reinterpret_cast<const float4*>(a.tw), tid, S_::THREADS);
    for (int i = tid; i < N; i += S_::THREADS) {
        dx_s[i] = a.vd[0][i];
        dy_s[i] = a.vd[1][i];
    }
    if (tid == 0) {
        mbar_init(bar, 1);      // rows 0..15 (into S)
        mbar_init(bar + 1, 1);  // rows 16..31 (into X)
    }
    __syncthreads();
    const cx<T>* twp = reinterpret_cast<const cx<T>*>(tws);
    pdl_wait();

    const unsigned row_bytes = (unsigned)(N * sizeof(cx<T>));
    // rows [r0, r0 + 16) of this CTA's slice of plane z land in `dst` at a
    // line stride of `stride` elements, completing on mbarrier b; the first
    // warp issues one bulk copy per row
    auto land_rows = [&](long z, int r0, cx<T>* dst, int stride, uint64_t* b) {
        if (tid < 32) {
            // order earlier generic-proxy accesses to dst before the bulk
            // copies (async proxy) that overwrite it
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (tid == 0)
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                             ::"r"(smem_addr(b)), "r"(row_bytes * LPR) : "memory");
            __syncwarp();
            if (tid < LPR) {
                const cx<T>* src = in + (size_t)z * plane + (size_t)(rank * RPC + r0 + tid) * N;
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], "
                    "[%1], %2, [%3];" ::"r"(smem_addr(dst + tid * stride)),
                    "l"(src), "r"(row_bytes), "r"(smem_addr(b))
                    : "memory");
            }
        }
    };

    // row phase: thread rt of line rl (rows rl and LPR + rl); column phase:
    // thread ct of column cc (columns cc and LPR + cc of this CTA's 32)
    const int rt = tid % P, rl = tid / P;
    const int cc = tid % LPR, ct = tid / LPR;
    auto row_sync = [] { __syncwarp(); };
    auto col_sync = [] { __syncthreads(); };
    const unsigned x_addr = smem_addr(X);

    KSum acc{0.0, 0.0};
    bool ok = true;
    unsigned par0 = 0, par1 = 0;
    long z = cluster_index();
    if (z < nz) land_rows(z, 0, Sx, S_::SLS, bar);
    cluster_arrive();  // X is free (pairs with the first wait below)
    for (; z < nz; z += zstep) {
        cluster_wait();  // the cluster has finished reading the previous plane's X
        if constexpr (LPR < RPC) land_rows(z, LPR, X + LPR * S_::LSR, S_::LSR, bar + 1);

        // ---- row phase (x lines): rows 0..15 from S, then rows 16..31 from
        // their X slots; the transforms exchange through S
        const double sc = (!INV && a.ops[0]) ? *a.scale_in : 1.0;
#pragma unroll 1
        for (int rd = 0; rd < RPC / LPR; ++rd) {
            const int row = rd * LPR + rl;
            cx<T>* xr = X + row * S_::LSR;
            const cx<T>* src = rd == 0 ? Sx + rl * S_::SLS : xr;
            ok &= mbar_wait(bar + rd, rd == 0 ? par0 : par1, kPlaneWaitPolls);
            cx<T> v[E];
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = src[L::index(rt, e)];
            __syncthreads();  // every row's landed values are in registers
            cx<T>* srow = Sx + rl * S_::SLS;
            if constexpr (!INV) {
                const int y = (int)rank * RPC + row;
                const cx<double> lf =
                    cscale(cmul(ld2(a.vfac[1], y), ld2(a.vfac[2], (int)z)), sc);
                // the pending scale is folded into the factor, so the density
                // of the unscaled values takes it squared
                op_vhalf_f32<L>(v, rt, dx_s, line_delta(lf), a, a.nl_coef * sc * sc);
                L::template forward<true>(v, rt, srow, twp, row_sync);
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
                L::template forward<true>(v, rt, srow, twp, row_sync);
#pragma unroll
                for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
            }
#pragma unroll
            for (int e = 0; e < E; ++e) xr[smem_phys(L::index(rt, e))] = v[e];
        }
        par0 ^= 1u;
        if constexpr (LPR < RPC) par1 ^= 1u;
        cluster_arrive();
        cluster_wait();  // every CTA's X holds this plane's rows

        // ---- column phase (y lines): element y of column x sits in CTA
        // y / 32, row y % 32, of X
#pragma unroll 1
        for (int rd = 0; rd < RPC / LPR; ++rd) {
            const int x_col = (int)rank * RPC + rd * LPR + cc;
            const int col_off = smem_phys(x_col);
            cx<T> v[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int y = L::index(ct, e);
                const unsigned la =
                    x_addr + (unsigned)(((y % RPC) * S_::LSR + col_off) * (int)sizeof(cx<T>));
                v[e] = dsmem_load<T>(dsmem_map(la, (unsigned)(y / RPC)));
            }
            const bool last = rd == RPC / LPR - 1;
            if (last) cluster_arrive();  // done reading X
            cx<T>* scol = Sx + cc * S_::LSC;
            if constexpr (INV) {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
            }
            L::template forward<true>(v, ct, scol, twp, col_sync);
            // S is free again (the transform ends with a block barrier): the
            // next plane's first rows land there while this one finishes
            if (last && z + zstep < nz) land_rows(z + zstep, 0, Sx, S_::SLS, bar);
            if constexpr (INV) {
#pragma unroll
                for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
                const cx<double> lf = cmul(ld2(a.vfac[0], x_col), ld2(a.vfac[2], (int)z));
                op_vhalf_f32<L>(v, ct, dy_s, line_delta(lf), a, a.nl_coef);
                if (a.red.kind == RED_NORM) op_norm_f32<E>(v, acc);
            }
            cx<T>* o = out + (size_t)z * plane + x_col;
#pragma unroll
            for (int e = 0; e < E; ++e) o[(size_t)L::index(ct, e) * N] = v[e];
        }
    }
    cluster_wait();  // no CTA leaves while another may still read its X
    if (!ok && a.err) atomicExch(a.err, 1);
    pdl_launch_dependents();
    if (INV && a.red.kind != RED_NONE) {
        __syncthreads();
        grid_reduce_finish(acc, reinterpret_cast<double*>(Sx), a.red, gridDim.x, blockIdx.x);
    }
}

}  // namespace gpue
