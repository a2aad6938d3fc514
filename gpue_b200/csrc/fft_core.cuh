// fft_core.cuh -- the line FFT engine used by every pass kernel.
//
// A "line" is one 1D transform of length N along one axis of the field.  P
// threads cooperate on a line; each holds E = N/P complex values in registers.
// The transform is a Stockham autosort FFT (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC'08)
// with a palindromic radix sequence (RA, RA) or (RA, RB, RA):
//
//   stage s, radix R, Ns = product of earlier radices, j = t + P*q:
//     inputs   x[j + r*N/R]             (r < R, read from registers/smem)
//     twiddle  W_{Ns R}^{(j mod Ns) r}  (from a per-N table W_N^k)
//     R-point DFT in registers
//     outputs  y[(j/Ns)*Ns*R + (j mod Ns) + r*Ns]
//
// Stage 0 reads straight from the registers loaded from HBM, the last stage
// leaves its outputs in registers, and the middle exchanges go through shared
// memory (one 8- or 16-byte access per element).  Because the sequence is
// palindromic, the register layout before and after a transform is the same
// ("layout D": register e = q*RA + r holds element t + P*q + r*N/RA), so
// forward and inverse transforms and pointwise phase multiplies chain inside
// one kernel without extra data movement, and global loads/stores in layout D
// are coalesced across threads.
//
// Transforms are unnormalised with cuFFT's signs (forward exp(-2 pi i jk/N)),
// which is what GPUE's evolve() uses before its 1/sqrt(N) scalarMult; the
// passes fold the 1/N of each forward/inverse pair into a phase factor.  The
// inverse is conj(F(conj(x))): either conjugated around the forward body, or
// the same body with every twiddle and +-i conjugated (forward<.., true>),
// which gives the same values without the conjugation sweeps.

#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include "twiddles.h"

namespace gpue {

template <typename T>
struct alignas(2 * sizeof(T)) cx {
    T x, y;
};

template <typename T>
__device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ cx<T> cscale(cx<T> a, T s) { return {a.x * s, a.y * s}; }
template <typename T>
__device__ __forceinline__ cx<T> cconj(cx<T> a) { return {a.x, -a.y}; }
// multiply by -i, by +i
template <typename T>
__device__ __forceinline__ cx<T> mul_mi(cx<T> a) { return {a.y, -a.x}; }
template <typename T>
__device__ __forceinline__ cx<T> mul_pi(cx<T> a) { return {-a.y, a.x}; }

// Complex64 sums and differences as packed FP32x2 operations (sm_100: one
// instruction for both components).  Each component is rounded exactly as
// the scalar operation rounds it (a - b is formed as b * -1 + a, whose
// product is exact), so results do not change, only the instruction count.
__device__ __forceinline__ float2 f2(cx<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ cx<float> c2(float2 a) { return {a.x, a.y}; }
__device__ __forceinline__ cx<float> operator+(cx<float> a, cx<float> b) {
    return c2(__fadd2_rn(f2(a), f2(b)));
}
__device__ __forceinline__ cx<float> operator-(cx<float> a, cx<float> b) {
    return c2(__ffma2_rn(f2(b), make_float2(-1.f, -1.f), f2(a)));
}

// Complex64 twiddles are carried as a pair of floats, hi + lo, equal to the
// FP64 twiddle to about 2^-48.  A single rounded float has |W|^2 = 1 - O(1e-8)
// on average (the rounding of cos and sin is not magnitude-neutral), which
// repeated transforms turn into a slow systematic drift of the state; with the
// pair the product a*W carries only the rounding of the arithmetic, which is
// unbiased.  It costs two fused multiply-adds per real output.
constexpr bool kSplitTwiddles = true;       // stage twiddles (per-N table)
constexpr bool kSplitConstTwiddles = true;  // butterfly constants

// a * (hi + lo)
__device__ __forceinline__ cx<float> cmul_split(cx<float> a, cx<float> hi, cx<float> lo) {
    const float tx = fmaf(a.x, lo.x, -a.y * lo.y);
    const float ty = fmaf(a.x, lo.y, a.y * lo.x);
    return {fmaf(a.x, hi.x, fmaf(-a.y, hi.y, tx)), fmaf(a.x, hi.y, fmaf(a.y, hi.x, ty))};
}
// a * conj(hi + lo), the product cmul_split forms on conjugated values,
// conjugated (the same operations with the signs moved: bit-identical)
__device__ __forceinline__ cx<float> cmul_split_conj(cx<float> a, cx<float> hi, cx<float> lo) {
    const float tx = fmaf(a.x, lo.x, a.y * lo.y);
    const float ty = fmaf(-a.x, lo.y, a.y * lo.x);
    return {fmaf(a.x, hi.x, fmaf(a.y, hi.y, tx)), fmaf(-a.x, hi.y, fmaf(a.y, hi.x, ty))};
}
// The same product for a constant twiddle, as four packed FP32x2 operations
// in the same order (bit-identical to cmul_split): the constant pairs
// (lo.x, lo.y), (-lo.y, lo.x), (-hi.y, hi.x), (hi.x, hi.y) need no shuffling
__device__ __forceinline__ cx<float> cmul_split_const(cx<float> a, float hx, float hy, float lx,
                                                      float ly) {
    const float2 ax = make_float2(a.x, a.x), ay = make_float2(a.y, a.y);
    float2 t = __fmul2_rn(ay, make_float2(-ly, lx));
    t = __ffma2_rn(ax, make_float2(lx, ly), t);
    t = __ffma2_rn(ay, make_float2(-hy, hx), t);
    return c2(__ffma2_rn(ax, make_float2(hx, hy), t));
}

// a * W_R^m, W_R = exp(-2 pi i / R), with exact shortcuts at multiples of pi/2
template <int R, int M, typename T>
__device__ __forceinline__ cx<T> tw_const(cx<T> a) {
    constexpr int m = ((M % R) + R) % R;
    if constexpr (m == 0) {
        return a;
    } else if constexpr (2 * m == R) {
        return {-a.x, -a.y};
    } else if constexpr (4 * m == R) {
        return mul_mi(a);
    } else if constexpr (4 * m == 3 * R) {
        return {-a.y, a.x};
    } else if constexpr (kSplitConstTwiddles && std::is_same<T, float>::value) {
        constexpr double c = tw_cos(R, m), s = -tw_sin(R, m);
        constexpr float ch = (float)c, sh = (float)s;
        constexpr float cl = (float)(c - (double)ch), sl = (float)(s - (double)sh);
        return cmul_split_const(a, ch, sh, cl, sl);
    } else if constexpr (8 * m == R || 8 * m == 3 * R || 8 * m == 5 * R || 8 * m == 7 * R) {
        constexpr T h = (T)0.70710678118654752440;
        constexpr double c = tw_cos(R, m);
        constexpr double s = tw_sin(R, m);
        constexpr T cs = c > 0 ? h : -h;
        constexpr T ss = s > 0 ? -h : h;  // W = c - i s
        return {cs * a.x - ss * a.y, cs * a.y + ss * a.x};
    } else {
        constexpr T c = (T)tw_cos(R, m);
        constexpr T s = (T)-tw_sin(R, m);
        return {c * a.x - s * a.y, c * a.y + s * a.x};
    }
}

// ---------------------------------------------------------- small DFTs --
// In-place R-point DFT of v[0..R-1] in registers, natural order: forward
// (exp(-2 pi i jk/R)), or with INV the inverse (exp(+2 pi i jk/R)), which
// equals conj(F(conj v)) operation for operation (every twiddle and +-i
// conjugated), so no conjugation pass is needed around it.

template <int R, typename T, bool INV = false>
struct SmallDFT;

template <typename T, bool INV>
struct SmallDFT<2, T, INV> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        cx<T> a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};

template <typename T, bool INV>
struct SmallDFT<3, T, INV> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        constexpr T c1 = (T)-0.5;
        constexpr T s1 = (T)-tw_sin(3, 1);
        cx<T> t1 = v[1] + v[2];
        cx<T> t2 = v[1] - v[2];
        cx<T> a = {v[0].x + c1 * t1.x, v[0].y + c1 * t1.y};
        cx<T> b;  // i*s1*t2 (forward), -i*s1*t2 (inverse)
        if constexpr (INV) b = {s1 * t2.y, -s1 * t2.x};
        else b = {-s1 * t2.y, s1 * t2.x};
        v[0] = v[0] + t1;
        v[1] = a + b;
        v[2] = a - b;
    }
};

template <typename T, bool INV>
struct SmallDFT<4, T, INV> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        cx<T> s02 = v[0] + v[2], d02 = v[0] - v[2];
        cx<T> s13 = v[1] + v[3];
        cx<T> d13 = INV ? mul_pi(v[1] - v[3]) : mul_mi(v[1] - v[3]);
        v[0] = s02 + s13;
        v[1] = d02 + d13;
        v[2] = s02 - s13;
        v[3] = d02 - d13;
    }
};

// Complex64: the four sums and differences packed, the +-i products as
// scalar component sums (the same values as the generic form)
template <bool INV>
struct SmallDFT<4, float, INV> {
    static __device__ __forceinline__ void run(cx<float>* v) {
        const cx<float> s02 = v[0] + v[2], d02 = v[0] - v[2];
        const cx<float> s13 = v[1] + v[3], d13 = v[1] - v[3];
        v[0] = s02 + s13;
        v[2] = s02 - s13;
        if constexpr (INV) {
            v[1] = {d02.x - d13.y, d02.y + d13.x};
            v[3] = {d02.x + d13.y, d02.y - d13.x};
        } else {
            v[1] = {d02.x + d13.y, d02.y - d13.x};
            v[3] = {d02.x - d13.y, d02.y + d13.x};
        }
    }
};

template <typename T, bool INV>
struct SmallDFT<5, T, INV> {
    static __device__ __forceinline__ void run(cx<T>* v) {
        constexpr T c1 = (T)tw_cos(5, 1), c2 = (T)tw_cos(5, 2);
        constexpr T s1 = (T)-tw_sin(5, 1);
        constexpr T s2 = (T)-tw_sin(5, 2);
        cx<T> a1 = v[1] + v[4], b1 = v[1] - v[4];
        cx<T> a2 = v[2] + v[3], b2 = v[2] - v[3];
        cx<T> r1 = {v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y};
        cx<T> r2 = {v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y};
        // i*(s1 b1 + s2 b2) and i*(s2 b1 - s1 b2); -i times the same (inverse)
        cx<T> i1, i2;
        if constexpr (INV) {
            i1 = {s1 * b1.y + s2 * b2.y, -(s1 * b1.x + s2 * b2.x)};
            i2 = {s2 * b1.y - s1 * b2.y, -(s2 * b1.x - s1 * b2.x)};
        } else {
            i1 = {-(s1 * b1.y + s2 * b2.y), s1 * b1.x + s2 * b2.x};
            i2 = {-(s2 * b1.y - s1 * b2.y), s2 * b1.x - s1 * b2.x};
        }
        v[0] = v[0] + a1 + a2;
        v[1] = r1 + i1;
        v[4] = r1 - i1;
        v[2] = r2 + i2;
        v[3] = r2 - i2;
    }
};

// Composite R = A*B: B DFTs of length A on stride-B subsequences, twiddles
// W_R^{b k1} (conjugated for the inverse), then A DFTs of length B;
// X[k1 + A*k2].
template <int R>
struct Split {
    static constexpr int A = (R % 4 == 0 && R != 8 && R != 4) ? 4
                             : (R % 2 == 0) ? 2
                             : (R % 3 == 0) ? 3
                                            : 5;
    static constexpr int B = R / A;
};

template <int R, typename T, bool INV>
struct SmallDFT {
    static constexpr int A = Split<R>::A;
    static constexpr int B = Split<R>::B;
    template <int b, int k1>
    static __device__ __forceinline__ void tw_one(cx<T> (&y)[B][A]) {
        y[b][k1] = tw_const<R, INV ? -(b * k1) : b * k1>(y[b][k1]);
    }
    template <int... I>
    static __device__ __forceinline__ void twiddle_all(cx<T> (&y)[B][A],
                                                       std::integer_sequence<int, I...>) {
        (tw_one<I / A, I % A>(y), ...);
    }
    static __device__ __forceinline__ void run(cx<T>* v) {
        cx<T> y[B][A];
#pragma unroll
        for (int b = 0; b < B; ++b) {
#pragma unroll
            for (int a = 0; a < A; ++a) y[b][a] = v[b + B * a];
            SmallDFT<A, T, INV>::run(y[b]);
        }
        twiddle_all(y, std::make_integer_sequence<int, B * A>{});
        cx<T> z[B];
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
#pragma unroll
            for (int b = 0; b < B; ++b) z[b] = y[b][k1];
            SmallDFT<B, T, INV>::run(z);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = z[k2];
        }
    }
};

// ------------------------------------------------------------ line FFT --

__host__ __device__ __forceinline__ constexpr int smem_phys(int i) { return i + (i >> 4); }

template <typename T, int N_, int RA, int RB, int P_, int RC = 0>
struct LineFFT {
    static constexpr int N = N_;
    static constexpr int P = P_;
    static constexpr int NS = RB == 0 ? 2 : RC == 0 ? 3 : 4;
    static constexpr int E = N / P;
    static_assert(NS == 2   ? N == RA * RA
                  : NS == 3 ? N == RA * RB * RA
                            : N == RA * RB * RC * RA,
                  "palindromic radix plan");
    static_assert((N / RA) % P == 0, "threads must divide the butterflies of the outer stages");
    static_assert(NS == 2 || (N / RB) % P == 0, "threads must divide the middle stages");
    static_assert(NS < 4 || (N / RC) % P == 0, "threads must divide the middle stages");
    // smem line stride in complex elements: one pad per 16, rounded to 16 and
    // offset by 4 so the lines a strided-pass warp touches (lanes c + C*t)
    // fall on distinct banks
    static constexpr int LS = ((smem_phys(N - 1) + 1 + 15) / 16) * 16 + 4;

    __host__ __device__ static constexpr int radix(int s) {
        return s == 0 || s == NS - 1 ? RA : s == 1 ? RB : RC;
    }
    __host__ __device__ static constexpr int ns_before(int s) {
        return s == 0 ? 1 : s == 1 ? RA : s == 2 ? RA * RB : RA * RB * RC;
    }

    // element index held by register e in layout D
    static __device__ __forceinline__ int index(int t, int e) {
        return t + P * (e / RA) + (e % RA) * (N / RA);
    }

    // The twiddles stage S > 0 multiplies by.  When few enough, they are
    // loaded into registers before the exchange that precedes the stage, so
    // their latency overlaps the shared-memory round trip; when P is a
    // multiple of Ns they depend on t only and one set serves every group.
    // Larger sets (long odd-radix plans) are read at use, as registers are
    // scarce there.
    // TWS: the twiddle table is in shared memory (plain loads), else global
    // (read-only cache)
    template <bool TWS>
    static __device__ __forceinline__ float4 tw4(const float4* p) {
        if constexpr (TWS) return *p;
        else return __ldg(p);
    }
    template <bool TWS>
    static __device__ __forceinline__ cx<T> tw1(const cx<T>* p) {
        if constexpr (TWS) return *p;
        else return *p;
    }

    // TWS tables are laid out per stage: stage S's twiddles W_{Ns R}^{jm r}
    // (jm = j mod Ns, 0 < r < R) at stage_base(S) + (r - 1) Ns + jm, so the
    // threads of a warp (consecutive jm) read consecutive entries.
    __host__ __device__ static constexpr int stage_base(int S) {
        int b = 0;
        for (int s = 1; s < S; ++s) b += (radix(s) - 1) * ns_before(s);
        return b;
    }
    static constexpr int kStageTableLen = stage_base(NS);
    // Fills the per-stage table (float4 (hi, lo) pairs or cx<T>) from the
    // per-N table W_N^k; threads tid of nthreads share the work.
    template <typename W>
    static __device__ __forceinline__ void build_stage_table(W* dst, const W* __restrict__ src,
                                                             int tid, int nthreads) {
        for (int i = tid; i < kStageTableLen; i += nthreads) {
            int S = 1;
            while (S + 1 < NS && i >= stage_base(S + 1)) ++S;
            const int Ns = ns_before(S), R = radix(S), off = i - stage_base(S);
            const int r = off / Ns + 1, jm = off % Ns;
            dst[i] = src[jm * r * (N / (Ns * R))];
        }
    }
    template <int S>
    static __device__ __forceinline__ int tw_index(int jm, int r) {
        return stage_base(S) + (r - 1) * ns_before(S) + jm;
    }

    template <int S, bool TWS = false>
    struct StageTw {
        static constexpr int R = radix(S);
        static constexpr int Ns = ns_before(S);
        static constexpr int G = N / (R * P);
        static constexpr int step = N / (Ns * R);
        static constexpr int NQ = (S > 0 && P % Ns == 0) ? 1 : G;
        // complex64 twiddles come as hi/lo pairs: entry k of the table is one
        // 16-byte (hi.x, hi.y, lo.x, lo.y), read with a single load
        static constexpr bool SPLIT = kSplitTwiddles && std::is_same<T, float>::value;
        static constexpr int WPER = SPLIT ? 2 : 1;
        static constexpr bool HOLD = NQ * (R - 1) * WPER <= 16;
        cx<T> w[HOLD ? NQ : 1][HOLD ? R - 1 : 1][WPER];
        const cx<T>* __restrict__ tw;
        int t;

        __device__ __forceinline__ void load(int t_, const cx<T>* __restrict__ tw_) {
            t = t_;
            tw = tw_;
            if constexpr (HOLD) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int jm = (t + P * q) % Ns;
#pragma unroll
                    for (int r = 1; r < R; ++r) {
                        const int k = TWS ? tw_index<S>(jm, r) : jm * r * step;
                        if constexpr (SPLIT) {
                            const float4 e = tw4<TWS>(reinterpret_cast<const float4*>(tw) + k);
                            w[q][r - 1][0] = cx<T>{e.x, e.y};
                            w[q][r - 1][WPER - 1] = cx<T>{e.z, e.w};
                        } else {
                            w[q][r - 1][0] = tw1<TWS>(tw + k);
                        }
                    }
                }
            }
        }
        // a times the twiddle (INV: its conjugate)
        template <bool INV>
        __device__ __forceinline__ cx<T> twmul(cx<T> a, cx<T> hi, cx<T> lo) const {
            if constexpr (SPLIT) {
                if constexpr (INV) return cmul_split_conj(a, hi, lo);
                else return cmul_split(a, hi, lo);
            } else {
                return cmul(a, INV ? cconj(hi) : hi);
            }
        }
        template <bool INV = false>
        __device__ __forceinline__ cx<T> mul(cx<T> a, int q, int r) const {
            if constexpr (HOLD) {
                const int qq = NQ == 1 ? 0 : q;
                return twmul<INV>(a, w[qq][r - 1][0], w[qq][r - 1][WPER - 1]);
            } else {
                const int k = TWS ? tw_index<S>((t + P * q) % Ns, r)
                                  : ((t + P * q) % Ns) * r * step;
                if constexpr (SPLIT) {
                    const float4 e = tw4<TWS>(reinterpret_cast<const float4*>(tw) + k);
                    return twmul<INV>(a, cx<T>{e.x, e.y}, cx<T>{e.z, e.w});
                } else {
                    const cx<T> e = tw1<TWS>(tw + k);
                    return twmul<INV>(a, e, e);
                }
            }
        }
    };

    template <int S, bool TWS = false, bool INV = false>
    static __device__ __forceinline__ void compute(cx<T> (&v)[E], const StageTw<S, TWS>* w) {
        constexpr int R = radix(S);
        constexpr int G = N / (R * P);
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if constexpr (S > 0) {
#pragma unroll
                for (int r = 1; r < R; ++r)
                    v[q * R + r] = w->template mul<INV>(v[q * R + r], q, r);
            }
            SmallDFT<R, T, INV>::run(&v[q * R]);
        }
    }

    // Write stage S's outputs to smem, sync, read stage S+1's inputs, sync.
    template <int S, typename Sync>
    static __device__ __forceinline__ void exchange(cx<T> (&v)[E], int t, cx<T>* sl, Sync sync) {
        constexpr int R = radix(S);
        constexpr int Ns = ns_before(S);
        constexpr int G = N / (R * P);
#pragma unroll
        for (int q = 0; q < G; ++q) {
            const int j = t + P * q;
            const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
            for (int r = 0; r < R; ++r) sl[smem_phys(base + r * Ns)] = v[q * R + r];
        }
        sync();
        constexpr int R2 = radix(S + 1);
        constexpr int G2 = N / (R2 * P);
#pragma unroll
        for (int q = 0; q < G2; ++q) {
            const int j = t + P * q;
#pragma unroll
            for (int r = 0; r < R2; ++r) v[q * R2 + r] = sl[smem_phys(j + r * (N / R2))];
        }
        sync();
    }

    // One stage after the first: its twiddles are requested before the
    // exchange, so their latency overlaps the shared-memory round trip.
    template <int S, bool TWS, bool INV, typename Sync>
    static __device__ __forceinline__ void stage(cx<T> (&v)[E], int t, cx<T>* sl,
                                                 const cx<T>* __restrict__ tw, Sync sync) {
        StageTw<S, TWS> w;
        w.load(t, tw);
        exchange<S - 1>(v, t, sl, sync);
        compute<S, TWS, INV>(v, &w);
    }

    // Unnormalised DFT of the line: forward, or with INV the inverse with
    // conjugated twiddles (the same values as conjugating around the
    // forward transform, without the two conjugation sweeps).  TWS: tw points
    // to the per-stage table (build_stage_table) in shared memory.
    template <bool TWS = false, bool INV = false, typename Sync>
    static __device__ __forceinline__ void forward(cx<T> (&v)[E], int t, cx<T>* sl,
                                                   const cx<T>* __restrict__ tw, Sync sync) {
        compute<0, TWS, INV>(v, static_cast<const StageTw<0, TWS>*>(nullptr));
        stage<1, TWS, INV>(v, t, sl, tw, sync);
        if constexpr (NS >= 3) stage<2, TWS, INV>(v, t, sl, tw, sync);
        if constexpr (NS >= 4) stage<3, TWS, INV>(v, t, sl, tw, sync);
    }
};

}  // namespace gpue
