// pass.cuh -- one full-field read+write pass over lines of one axis.
//
// A pass walks tiles of C lines (rows for axis 0; C adjacent columns for the
// strided axes 1 and 2, so each row segment is at least one 32-byte sector),
// loads a tile into registers, runs a short program of operations, and
// stores it back.  The operations are the pieces of GPUE's split step
// (src/evolution.cu:727-870), fused so each pass touches memory once:
//
//   OP_SCALE   psi *= deferred renormalisation factor (parSum and
//              scalarDiv_wfcNorm, src/split_op.cu:83-129, applied by the next
//              pass that reads the field)
//   OP_VHALF   psi *= exp(-(V + gN|psi|^2) Dt/(2 hbar))        imaginary time
//              psi *= exp(-i(V + gN|psi|^2) Dt/(2 hbar))       real time
//              (cMultDensity, src/kernels.cu:365-388; cMult without -s)
//   OP_FFT_F / OP_FFT_I   unnormalised 1D DFT along the pass axis
//              (cufftExecZ2Z, src/evolution.cu:758,774)
//   OP_KPHASE  psi *= exp(-K Dt/hbar) / exp(-i K Dt/hbar) times 1/N, the
//              product of GPUE's two 1/sqrt(N) scalarMults
//              (K = hbar^2/(2m)|p|^2, src/operators.cu:460-469, 1081-1103)
//   OP_GAUGE   psi *= exp(-A_a p_a gdt) / exp(-i A_a p_a dt) times 1/n along
//              the pass axis (apply_gauge, src/evolution.cu:5-257; aux_fields
//              src/operators.cu:1089-1110)
//   OP_NORM    accumulate sum |psi|^2 (FP64, compensated) -> renorm factor
//   OP_EKIN    accumulate sum K |psi_k|^2 (FP64, compensated)
//
// V and K are separable per axis for the harmonic trap with the rotation
// gauge (V = Vx(x)+Vy(y)+Vz(z) including m|A|^2/2), so their factors come from
// per-axis FP64 tables.  Every phase factor is formed and applied in FP64 and
// real-time factors are normalised to unit modulus before the product is
// rounded back to the storage type: a complex64 factor rounded once and
// reused every step would otherwise grow or shrink the norm systematically.

#pragma once

#include <type_traits>

#include "ast_eval.cuh"
#include "fft_core.cuh"

namespace gpue {

enum PassOp : int {
    OP_NONE = 0,
    OP_FFT_F = 1,
    OP_FFT_I = 2,
    OP_SCALE = 3,
    OP_VHALF = 4,
    OP_KPHASE = 5,
    OP_GAUGE = 6,
    OP_NORM = 7,
    OP_EKIN = 8,
};

constexpr int kMaxOps = 8;

enum RedKind : int { RED_NONE = 0, RED_NORM = 1, RED_SUM = 2 };

// A grid-wide FP64 reduction: every CTA writes a compensated partial, the last
// CTA to finish sums them in index order and writes the result.
struct RedArgs {
    int kind;               // RED_NONE / RED_NORM / RED_SUM
    double2* partials;      // [gridDim.x] (sum, compensation)
    unsigned* counter;      // zero between reductions; reset by the last CTA
    double* out;            // RED_NORM: sqrt(*target / sum); RED_SUM: sum
    const double* target;   // RED_NORM target sum |psi|^2
};

struct PassArgs {
    const void* in;
    void* out;
    int axis;  // 0: x rows (contiguous), 1: y lines (stride nx), 2: z lines
    int nx, ny, nz;
    long ntiles;  // tiles of C lines
    int nops;
    int ops[kMaxOps];
    int store;   // write the lines back
    int gstate;  // 0 imaginary time, 1 real time
    int gpe;     // nonlinear term on
    double nl_coef;     // gN * (Dt/2) / hbar
    double kscale;      // folded into OP_KPHASE (1/N)
    double gscale;      // folded into OP_GAUGE (1/n of this axis)
    double gauge_coef;  // A_axis = gauge_coef * pos[gauge_src][.]
    int gauge_src;      // axis whose coordinate A_axis depends on
    double gauge_dt;    // gdt * ramp exponent (imaginary) or dt (real)
    double dmom;        // momentum spacing dp of the pass axis
    double kin_coef;    // hbar^2 / (2 m), for OP_EKIN
    const double2* vfac[3];  // per-axis V half-step factor (FP64)
    const double2* kfac[3];  // per-axis kinetic factor (FP64)
    const float2* vd[3];     // complex64 form: the V/2 factor minus 1, rounded once
    const float2* kd[3];     // complex64 form: the kinetic factor minus 1
    const double* pos[3];
    const double* mom[3];
    const void* tw;  // W_N^k for this axis: cx<double>[N], or (hi, lo) float pairs [N]
    RedArgs red;
    const double* scale_in;   // OP_SCALE factor
    const double* kscale_in;  // optional extra OP_KPHASE factor (real-time norm guard)
    // Extended forms (kernels built with EXT only): full-field tables of real
    // V and A (GPUE's static param-file fields, find_field at t = 0) and
    // time-dependent expressions evaluated per point and step at (i dx, j dy,
    // k dz, t) as evolve()'s AST kernels do.
    const double* vtab;      // V(g), replaces the separable V
    const double* atab[3];   // A_axis(g), replaces the rotation gauge
    const AstInstr* prog_v;  // time-dependent V
    const AstInstr* prog_k;  // time-dependent K
    const AstInstr* prog_a[3];
    int nprog_v, nprog_k, nprog_a[3];
    double time;             // Dt * step
    double step_dt;          // Dt
    double grid_d[3];        // dx, dy, dz as evolve() passes them (1 for absent axes)
    double hbar;
    const int* active;       // batched solves: 0 once converged (skip the tiles)
    int* err;                // plane passes: set non-zero when a bounded wait gave up
};

// Work counters of the TMA tile-stream passes (tstream.cuh); zero between
// launches (the last CTA of each launch clears them).
struct XYCounters {
    unsigned long long* ticket;  // next ticket
    unsigned* finish;            // CTAs finished
    int* done_x;                 // [nz] x-tiles stored per plane (XY pass)
    int lag;                     // XY pass: planes between a plane's x-tiles and y-tiles
    int wait_extra;              // XY pass: 0; > 0 only to test the bounded plane wait
};

// ------------------------------------------------------- FP64 reductions --

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

struct KSum {
    double s, c;
    __device__ __forceinline__ void add(double v) {
        double t, e;
        two_sum(s, v, t, e);
        s = t;
        c += e;
    }
    __device__ __forceinline__ void merge(double os, double oc) {
        double t, e;
        two_sum(s, os, t, e);
        s = t;
        c += oc + e;
    }
};

// Block-wide compensated reduction; result valid in thread 0.  `scratch`
// needs 2*(blockDim/32) doubles.
__device__ __forceinline__ KSum block_reduce(KSum k, double* scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double os = __shfl_down_sync(0xffffffffu, k.s, o);
        double oc = __shfl_down_sync(0xffffffffu, k.c, o);
        k.merge(os, oc);
    }
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if ((threadIdx.x & 31) == 0) {
        scratch[2 * w] = k.s;
        scratch[2 * w + 1] = k.c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum r{scratch[0], scratch[1]};
        for (int i = 1; i < nw; ++i) r.merge(scratch[2 * i], scratch[2 * i + 1]);
        k = r;
    }
    return k;
}

// Write this block's partial; the last block to arrive reduces all partials in
// index order (deterministic) and writes the result.  All threads call it.
// nparts CTAs take part; this one writes partial `idx`.
__device__ __forceinline__ void grid_reduce_finish(KSum k, double* scratch, const RedArgs& a,
                                                   unsigned nparts, unsigned idx) {
    __shared__ unsigned s_last;
    k = block_reduce(k, scratch);
    if (threadIdx.x == 0) {
        a.partials[idx] = make_double2(k.s, k.c);
        __threadfence();
        unsigned prev = atomicAdd(a.counter, 1u);
        s_last = (prev == nparts - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        KSum t{0.0, 0.0};
        for (unsigned i = threadIdx.x; i < nparts; i += blockDim.x) {
            double2 p = __ldcg(a.partials + i);
            t.merge(p.x, p.y);
        }
        __syncthreads();
        t = block_reduce(t, scratch);
        if (threadIdx.x == 0) {
            double sum = t.s + t.c;
            if (a.kind == RED_NORM)
                a.out[0] = sqrt(*a.target / sum);
            else
                a.out[0] = sum;
            *a.counter = 0u;
        }
    }
}

// ------------------------------------------------------------- helpers --

__device__ __forceinline__ cx<double> ld2(const double2* p, int i) {
    const double2 v = p[i];
    return {v.x, v.y};
}

// psi * f with f in FP64; for complex64 the product is formed in FP64 and
// rounded once.
template <typename T>
__device__ __forceinline__ cx<T> apply(cx<T> v, cx<double> f) {
    if constexpr (std::is_same<T, double>::value) {
        return cmul(v, f);
    } else {
        const double x = v.x, y = v.y;
        return cx<T>{(T)(x * f.x - y * f.y), (T)(x * f.y + y * f.x)};
    }
}

template <typename T>
__device__ __forceinline__ cx<double> unit_phase(double a);

// exp(-i a) for |a| < 1/16 by its Taylor series (truncation error below
// a^9/9! < 4e-17, so |result| = 1 to FP64 accuracy), no branch
__device__ __forceinline__ cx<double> taylor_phase(double a) {
    const double a2 = a * a;
    const double s = a * (1.0 - a2 * (1.0 / 6.0 - a2 * (1.0 / 120.0 - a2 * (1.0 / 5040.0))));
    const double c =
        1.0 - a2 * (0.5 - a2 * (1.0 / 24.0 - a2 * (1.0 / 720.0 - a2 * (1.0 / 40320.0))));
    return {c, -s};
}

// exp(-i a): the Taylor series for |a| < 1/16, else sincos
template <typename T>
__device__ __forceinline__ cx<double> small_phase(double a) {
    if (fabs(a) < 0.0625) return taylor_phase(a);
    return unit_phase<T>(a);
}

template <typename T>
__device__ __forceinline__ double decay(double a);

// exp(-a) for |a| < 1/16 by its Taylor series (truncation error below
// a^10/10! < 5e-19), no branch
__device__ __forceinline__ double taylor_decay(double a) {
    double r = 1.0 / 362880.0;
    r = 1.0 / 40320.0 - a * r;
    r = 1.0 / 5040.0 - a * r;
    r = 1.0 / 720.0 - a * r;
    r = 1.0 / 120.0 - a * r;
    r = 1.0 / 24.0 - a * r;
    r = 1.0 / 6.0 - a * r;
    r = 0.5 - a * r;
    r = 1.0 - a * r;
    return 1.0 - a * r;
}

// exp(-a): the Taylor series for |a| < 1/16, else exp
template <typename T>
__device__ __forceinline__ double small_decay(double a) {
    if (fabs(a) < 0.0625) return taylor_decay(a);
    return decay<T>(a);
}

// exp(-i a) with unit modulus to FP64 accuracy
template <typename T>
__device__ __forceinline__ cx<double> unit_phase(double a) {
    if constexpr (std::is_same<T, double>::value) {
        double s, c;
        sincos(-a, &s, &c);
        return {c, s};
    } else {
        float s, c;
        sincosf((float)-a, &s, &c);
        const double cd = c, sd = s;
        const double k = 1.5 - 0.5 * (cd * cd + sd * sd);  // one Newton step to |f| = 1
        return {cd * k, sd * k};
    }
}

template <typename T>
__device__ __forceinline__ double decay(double a) {
    if constexpr (std::is_same<T, double>::value) return exp(-a);
    else return (double)expf((float)-a);
}

// OP_VHALF with separable factors: psi *= fa[k] * lf * (nonlinear factor),
// fa the pass axis' FP64 V/2 factors, lf the product of the other axes' at the
// line.  The nonlinear angle gN|psi|^2 Dt/(2 hbar) is almost always below 1/16,
// where a Taylor series is exact to FP64: that is decided once for the
// thread's values (an FP32 estimate with margin), so the unrolled loops have
// no branch and the values' FP64 chains interleave.
template <typename T, class L>
__device__ __forceinline__ void op_vhalf_sep(cx<T> (&v)[L::E], int t, const double2* fa,
                                             cx<double> lf, const PassArgs& a) {
    constexpr int E = L::E;
    bool small = true;
    if (a.gpe) {
        const float nl = (float)a.nl_coef;
        float m = 0.f;
#pragma unroll
        for (int e = 0; e < E; ++e)
            m = fmaxf(m, fabsf(nl * ((float)v[e].x * (float)v[e].x +
                                     (float)v[e].y * (float)v[e].y)));
        small = m < 0.06f;
    }
    if (!a.gpe) {
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = apply(v[e], cmul(ld2(fa, L::index(t, e)), lf));
    } else if (small && a.gstate == 0) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double gd = a.nl_coef * ((double)v[e].x * v[e].x + (double)v[e].y * v[e].y);
            const cx<double> f = cmul(ld2(fa, L::index(t, e)), lf);
            v[e] = apply(v[e], cscale(f, taylor_decay(gd)));
        }
    } else if (small) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double gd = a.nl_coef * ((double)v[e].x * v[e].x + (double)v[e].y * v[e].y);
            const cx<double> f = cmul(ld2(fa, L::index(t, e)), lf);
            v[e] = apply(v[e], cmul(f, taylor_phase(gd)));
        }
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            cx<double> f = cmul(ld2(fa, L::index(t, e)), lf);
            const double gd = a.nl_coef * ((double)v[e].x * v[e].x + (double)v[e].y * v[e].y);
            if (a.gstate == 0) f = cscale(f, small_decay<T>(gd));
            else f = cmul(f, small_phase<T>(gd));
            v[e] = apply(v[e], f);
        }
    }
}

// OP_NORM: the thread's E terms summed in plain FP64 (relative error
// ~E * 2^-53), entering the compensated sum once per line.
template <typename T, int E>
__device__ __forceinline__ void op_norm(const cx<T> (&v)[E], KSum& acc) {
    double part = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const double re = (double)v[e].x, im = (double)v[e].y;
        part += re * re + im * im;
    }
    acc.add(part);
}

// ------------------------------------------------ complex64 phase factors --
//
// The complex64 form carries each factor f as d = f - 1, formed in FP64 (or
// higher) and rounded once to FP32, and applies it as psi + d*psi: the small
// correction d*psi is formed in FP32 and added with one rounding of psi's
// magnitude, which is as accurate as an FP64 product rounded once and keeps
// |f| = 1 of a real-time factor to FP32 round-off relative to |d|, with no
// systematic growth.  Products of separable factors combine as
// (1 + a)(1 + b) - 1 = a + b + a*b (no cancellation: the angles of one
// factor kind share a sign).

__device__ __forceinline__ float2 dmul(float2 a, float2 b) {
    float rx = a.x + b.x, ry = a.y + b.y;
    rx = fmaf(a.x, b.x, fmaf(-a.y, b.y, rx));
    ry = fmaf(a.x, b.y, fmaf(a.y, b.x, ry));
    return {rx, ry};
}
// psi + d*psi
__device__ __forceinline__ cx<float> dapply(cx<float> v, float2 d) {
    const float cx_ = fmaf(d.x, v.x, -d.y * v.y);
    const float cy_ = fmaf(d.x, v.y, d.y * v.x);
    return {v.x + cx_, v.y + cy_};
}
// psi + d*psi for a real d
__device__ __forceinline__ cx<float> dapply_re(cx<float> v, float d) {
    return {fmaf(d, v.x, v.x), fmaf(d, v.y, v.y)};
}
// f - 1 of an FP64 factor f near 1, rounded to FP32
__device__ __forceinline__ float2 line_delta(cx<double> f) {
    return {(float)(f.x - 1.0), (float)f.y};
}
__device__ __forceinline__ float2 ldf2(const float2* p, int i) { return p[i]; }

// exp(-i p) - 1 and exp(-p) - 1 for |p| < 1/16 by their Taylor series in
// FP32 (truncation below 2^-24 relative)
__device__ __forceinline__ float2 nl_phase_delta(float p) {
    const float p2 = p * p;
    const float sn = p * fmaf(-p2 * (1.f / 6.f), fmaf(-p2, 1.f / 20.f, 1.f), 1.f);
    const float cm = -0.5f * p2 * fmaf(-p2 * (1.f / 12.f), fmaf(-p2, 1.f / 30.f, 1.f), 1.f);
    return {cm, -sn};
}
__device__ __forceinline__ float nl_decay_delta(float p) {
    float r = fmaf(-p, 1.f / 120.f, 1.f / 24.f);
    r = fmaf(-p, r, 1.f / 6.f);
    r = fmaf(-p, r, 0.5f);
    r = fmaf(-p, r, 1.f);
    return -p * r;
}
// the same for any p, in FP64 from the FP64 angle, rounded once
__device__ __forceinline__ float2 nl_phase_delta64(double p) {
    double s, c;
    sincos(p, &s, &c);
    const double h = sin(0.5 * p);
    return {(float)(-2.0 * h * h), (float)(-s)};
}
__device__ __forceinline__ float nl_decay_delta64(double p) { return (float)expm1(-p); }

// OP_VHALF, complex64, separable V: psi *= (1 + dl)(1 + dk[k]) * nonlinear
// factor, dl the other axes' factors at the line (minus 1).  nl64 is the
// nonlinear coefficient for the density of the values in v (a.nl_coef, times
// s^2 when a pending scale s is folded into dl instead of applied to v).
template <class L>
__device__ __forceinline__ void op_vhalf_f32(cx<float> (&v)[L::E], int t, const float2* dk,
                                             float2 dl, const PassArgs& a, double nl64) {
    constexpr int E = L::E;
    const float nl = (float)nl64;
    bool small = true;
    if (a.gpe) {
        float m = 0.f;
#pragma unroll
        for (int e = 0; e < E; ++e) m = fmaxf(m, fabsf(nl * fmaf(v[e].x, v[e].x, v[e].y * v[e].y)));
        small = m < 0.06f;
    }
    if (!a.gpe) {
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = dapply(v[e], dmul(dl, ldf2(dk, L::index(t, e))));
    } else if (small && a.gstate == 0) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float dv = dl.x + ldf2(dk, L::index(t, e)).x +
                             dl.x * ldf2(dk, L::index(t, e)).x;
            const float dn = nl_decay_delta(nl * fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
            v[e] = dapply_re(v[e], fmaf(dv, dn, dv + dn));
        }
    } else if (small) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float2 dn = nl_phase_delta(nl * fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
            v[e] = dapply(v[e], dmul(dmul(dl, ldf2(dk, L::index(t, e))), dn));
        }
    } else {
        // large nonlinear angles: the factor from the FP64 angle in FP64
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double p = nl64 * ((double)v[e].x * v[e].x + (double)v[e].y * v[e].y);
            const float2 dv = dmul(dl, ldf2(dk, L::index(t, e)));
            const float2 dn = a.gstate == 0 ? float2{nl_decay_delta64(p), 0.f}
                                            : nl_phase_delta64(p);
            v[e] = dapply(v[e], dmul(dv, dn));
        }
    }
}

// OP_KPHASE, complex64, separable K: psi *= s (1 + dl)(1 + dk[k]), s the
// real scalings (1/N, the norm guard)
template <class L>
__device__ __forceinline__ void op_kphase_f32(cx<float> (&v)[L::E], int t, const float2* dk,
                                              float2 dl, float s) {
#pragma unroll
    for (int e = 0; e < L::E; ++e) {
        const cx<float> w = dapply(v[e], dmul(dl, ldf2(dk, L::index(t, e))));
        v[e] = {w.x * s, w.y * s};
    }
}

// The same, with the k factors as (d.x, d.y, d.y, d.x) and the product of
// the line and k factors (dmul) and the real scaling as packed FP32x2
// operations in dmul's order: bit-identical to op_kphase_f32.
template <class L>
__device__ __forceinline__ void op_kphase_f32_packed(cx<float> (&v)[L::E], int t,
                                                     const float4* dk, float2 dl, float s) {
    const float2 lneg = make_float2(-dl.y, dl.y), lx = make_float2(dl.x, dl.x);
    const float2 ss = make_float2(s, s);
#pragma unroll
    for (int e = 0; e < L::E; ++e) {
        const float4 q = dk[L::index(t, e)];
        float2 d = __fadd2_rn(dl, make_float2(q.x, q.y));
        d = __ffma2_rn(lneg, make_float2(q.z, q.w), d);
        d = __ffma2_rn(lx, make_float2(q.x, q.y), d);
        const cx<float> w = dapply(v[e], d);
        const float2 r = __fmul2_rn(make_float2(w.x, w.y), ss);
        v[e] = {r.x, r.y};
    }
}

// OP_NORM, complex64: the thread's |psi|^2 summed in FP32 (relative error
// ~E 2^-24 per thread, unbiased), entering the FP64 compensated sum once
template <int E>
__device__ __forceinline__ void op_norm_f32(const cx<float> (&v)[E], KSum& acc) {
    float part = 0.f;
#pragma unroll
    for (int e = 0; e < E; ++e) part += fmaf(v[e].x, v[e].x, v[e].y * v[e].y);
    acc.add((double)part);
}

// ---------------------------------------------------------------- kernel --

constexpr int kMaxPassThreads = 256;

// Programmatic dependent launch: once a pass kernel's CTAs have finished
// their tiles, the next pass kernel in the stream may start launching (its
// CTAs become resident while this grid drains), and every pass kernel waits
// for the grid before it to complete -- with its memory visible -- before
// touching any data.  Both are no-ops for a kernel launched without the
// programmatic-serialization attribute.
__device__ __forceinline__ void pdl_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }


// C = blockDim.x / P lines per tile; CTAs walk tiles with a grid stride.
// make_complex (src/kernels.cu:165-187): 1 -> exp(-v), 2 -> exp(-i v)
__device__ __forceinline__ cx<double> make_complex_ev(double v, int type) {
    if (type == 1) return {exp(-v), 0.0};
    double s, c;
    sincos(-v, &s, &c);
    return {c, s};
}

// EXT: also the table and expression forms of the factor ops.
// Tiles t0, t0 + tstep, ... of one field; returns this thread's OP_NORM /
// OP_EKIN accumulation.
template <typename T, int N, int RA, int RB, int P, bool STRIDED, bool EXT, int RC = 0>
__device__ __forceinline__ KSum pass_tiles(const PassArgs& a, long t0, long tstep,
                                           unsigned char* smem_raw) {
    using L = LineFFT<T, N, RA, RB, P, RC>;
    constexpr int E = L::E;

    const int C = blockDim.x / P;
    int c, t;
    if constexpr (STRIDED) {
        c = threadIdx.x % C;
        t = threadIdx.x / C;
    } else {
        t = threadIdx.x % P;
        c = threadIdx.x / P;
    }
    cx<T>* sl = reinterpret_cast<cx<T>*>(smem_raw) + c * L::LS;

    auto sync = [] {
        if constexpr (STRIDED || P > 32) __syncthreads();
        else __syncwarp();
    };

    const cx<T>* __restrict__ tw = reinterpret_cast<const cx<T>*>(a.tw);
    const long nxy = (long)a.nx * a.ny;
    KSum acc{0.0, 0.0};

    for (long tile = t0; tile < a.ntiles; tile += tstep) {
        const long line = tile * C + c;
        long base, stride;
        int xi = 0, yi = 0, zi = 0;  // line coordinates (the pass axis one is per element)
        if (a.axis == 0) {
            yi = (int)(line % a.ny);
            zi = (int)(line / a.ny);
            base = line * a.nx;
            stride = 1;
        } else if (a.axis == 1) {
            xi = (int)(line % a.nx);
            zi = (int)(line / a.nx);
            base = xi + zi * nxy;
            stride = a.nx;
        } else {
            xi = (int)(line % a.nx);
            yi = (int)(line / a.nx);
            base = line;
            stride = nxy;
        }

        cx<T> v[E];
        {
            const cx<T>* in = reinterpret_cast<const cx<T>*>(a.in) + base;
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = in[(long)L::index(t, e) * stride];
        }

        for (int o = 0; o < a.nops; ++o) {
            const int op = a.ops[o];
            switch (op) {
                case OP_FFT_F:
                case OP_FFT_I: {
                    const bool inv = (op == OP_FFT_I);
                    if (inv) {
#pragma unroll
                        for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
                    }
                    L::forward(v, t, sl, tw, sync);
                    if (inv) {
#pragma unroll
                        for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
                    }
                    break;
                }
                case OP_SCALE: {
                    const T s = (T)(*a.scale_in);
#pragma unroll
                    for (int e = 0; e < E; ++e) v[e] = cscale(v[e], s);
                    break;
                }
                case OP_VHALF: {
                    if constexpr (EXT) {
                        if (a.prog_v || a.vtab) {
                            // cMultDensity_ast (src/kernels.cu:391-422): V(x,t) with no
                            // dt factor; linear: ast_op_mult with the full Dt.  Static
                            // tables: the aux_fields factors of V(g).
                            const double* d = a.grid_d;
#pragma unroll
                            for (int e = 0; e < E; ++e) {
                                const int k = L::index(t, e);
                                cx<double> f;
                                if (a.prog_v) {
                                    const double px = (a.axis == 0 ? k : xi) * d[0];
                                    const double py = (a.axis == 1 ? k : yi) * d[1];
                                    const double pz = (a.axis == 2 ? k : zi) * d[2];
                                    const double val =
                                        ast_eval(a.prog_v, a.nprog_v, px, py, pz, a.time);
                                    f = make_complex_ev(a.gpe ? val : val * a.step_dt,
                                                        a.gstate + 1);
                                } else {
                                    const double V = a.vtab[base + (long)k * stride];
                                    const double ang = V * (a.step_dt / (2.0 * a.hbar));
                                    f = a.gstate == 0 ? cx<double>{small_decay<T>(ang), 0.0}
                                                      : small_phase<T>(ang);
                                }
                                if (a.gpe) {
                                    const double gd = a.nl_coef * ((double)v[e].x * v[e].x +
                                                                   (double)v[e].y * v[e].y);
                                    if (a.gstate == 0) f = cscale(f, small_decay<T>(gd));
                                    else f = cmul(f, small_phase<T>(gd));
                                }
                                v[e] = apply(v[e], f);
                            }
                            break;
                        }
                    }
                    cx<double> lf;
                    if (a.axis == 0) lf = cmul(ld2(a.vfac[1], yi), ld2(a.vfac[2], zi));
                    else if (a.axis == 1) lf = cmul(ld2(a.vfac[0], xi), ld2(a.vfac[2], zi));
                    else lf = cmul(ld2(a.vfac[0], xi), ld2(a.vfac[1], yi));
                    if constexpr (std::is_same<T, float>::value)
                        op_vhalf_f32<L>(v, t, a.vd[a.axis], line_delta(lf), a, a.nl_coef);
                    else
                        op_vhalf_sep<T, L>(v, t, a.vfac[a.axis], lf, a);
                    break;
                }
                case OP_KPHASE: {
                    if constexpr (EXT) {
                        if (a.prog_k) {
                            // ast_op_mult with the "k" expression at the position
                            // coordinates of the indices (src/evolution.cu:764-768)
                            const double* d = a.grid_d;
                            const double ks = a.kscale_in ? a.kscale * *a.kscale_in : a.kscale;
#pragma unroll
                            for (int e = 0; e < E; ++e) {
                                const int k = L::index(t, e);
                                const double px = (a.axis == 0 ? k : xi) * d[0];
                                const double py = (a.axis == 1 ? k : yi) * d[1];
                                const double pz = (a.axis == 2 ? k : zi) * d[2];
                                const double val =
                                    ast_eval(a.prog_k, a.nprog_k, px, py, pz, a.time);
                                v[e] = apply(v[e], cscale(make_complex_ev(val * a.step_dt,
                                                                          a.gstate + 1), ks));
                            }
                            break;
                        }
                    }
                    cx<double> lf;
                    if (a.axis == 0) lf = cmul(ld2(a.kfac[1], yi), ld2(a.kfac[2], zi));
                    else if (a.axis == 1) lf = cmul(ld2(a.kfac[0], xi), ld2(a.kfac[2], zi));
                    else lf = cmul(ld2(a.kfac[0], xi), ld2(a.kfac[1], yi));
                    const double ks = a.kscale_in ? a.kscale * *a.kscale_in : a.kscale;
                    if constexpr (std::is_same<T, float>::value) {
                        op_kphase_f32<L>(v, t, a.kd[a.axis], line_delta(lf), (float)ks);
                    } else {
                        lf = cscale(lf, ks);
                        const double2* fa = a.kfac[a.axis];
#pragma unroll
                        for (int e = 0; e < E; ++e)
                            v[e] = apply(v[e], cmul(ld2(fa, L::index(t, e)), lf));
                    }
                    break;
                }
                case OP_GAUGE: {
                    if constexpr (EXT) {
                        if (a.prog_a[a.axis] || a.atab[a.axis]) {
                            // ast_cmult multiplies by the raw A(x,t) (src/kernels.cu:
                            // 632-645); tables give exp(-A(g) p_k dt) per point
                            const double* d = a.grid_d;
                            const AstInstr* pr = a.prog_a[a.axis];
                            const double* mom = a.mom[a.axis];
#pragma unroll
                            for (int e = 0; e < E; ++e) {
                                const int k = L::index(t, e);
                                cx<double> f;
                                if (pr) {
                                    const double px = (a.axis == 0 ? k : xi) * d[0];
                                    const double py = (a.axis == 1 ? k : yi) * d[1];
                                    const double pz = (a.axis == 2 ? k : zi) * d[2];
                                    f = {ast_eval(pr, a.nprog_a[a.axis], px, py, pz, a.time), 0.0};
                                } else {
                                    const double ang =
                                        a.atab[a.axis][base + (long)k * stride] * mom[k] * a.gauge_dt;
                                    f = a.gstate == 0 ? cx<double>{small_decay<T>(ang), 0.0}
                                                      : small_phase<T>(ang);
                                }
                                v[e] = apply(v[e], cscale(f, a.gscale));
                            }
                            break;
                        }
                    }
                    // exp(-A p dt) / exp(-i A p dt) with p = m dp, m the signed
                    // frequency of index k (m = k - n for k >= n/2): geometric in
                    // k, so the factor of k = t + P q + r n/RA is
                    // W^t A^q B^r (times W^-n above n/2) with W = w(dp),
                    // A = W^P, B = W^(n/RA), formed in FP64.
                    const int src = a.gauge_src;
                    const int sidx = (src == 0) ? xi : (src == 1) ? yi : zi;
                    const double ang1 = a.gauge_coef * a.pos[src][sidx] * a.gauge_dt * a.dmom;
                    constexpr int QN = E / RA;
                    if (a.gstate == 0) {
                        const double wt = exp(-ang1 * t) * a.gscale;
                        const double wa = exp(-ang1 * P), wb = exp(-ang1 * (N / RA));
                        const double wn = exp(ang1 * N);
                        double aq = wt;
#pragma unroll
                        for (int q = 0; q < QN; ++q) {
                            double f = aq;
#pragma unroll
                            for (int r = 0; r < RA; ++r) {
                                const int e = q * RA + r;
                                const double ff = (t + P * q + r * (N / RA) >= N / 2) ? f * wn : f;
                                v[e] = apply(v[e], cx<double>{ff, 0.0});
                                f *= wb;
                            }
                            aq *= wa;
                        }
                    } else {
                        cx<double> wt = cscale(unit_phase<double>(ang1 * t), a.gscale);
                        const cx<double> wa = unit_phase<double>(ang1 * P);
                        const cx<double> wb = unit_phase<double>(ang1 * (N / RA));
                        const cx<double> wn = unit_phase<double>(-ang1 * N);
                        cx<double> aq = wt;
#pragma unroll
                        for (int q = 0; q < QN; ++q) {
                            cx<double> f = aq;
#pragma unroll
                            for (int r = 0; r < RA; ++r) {
                                const int e = q * RA + r;
                                const cx<double> ff =
                                    (t + P * q + r * (N / RA) >= N / 2) ? cmul(f, wn) : f;
                                v[e] = apply(v[e], ff);
                                f = cmul(f, wb);
                            }
                            aq = cmul(aq, wa);
                        }
                    }
                    break;
                }
                case OP_NORM:
                    if constexpr (std::is_same<T, float>::value) op_norm_f32<E>(v, acc);
                    else op_norm<T, E>(v, acc);
                    break;
                case OP_EKIN: {
                    double part = 0.0;
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const int k = L::index(t, e);
                        const double px = a.mom[0][a.axis == 0 ? k : xi];
                        const double py = a.mom[1][a.axis == 1 ? k : yi];
                        const double pz = a.mom[2][a.axis == 2 ? k : zi];
                        const double K = a.kin_coef * (px * px + py * py + pz * pz);
                        const double re = (double)v[e].x, im = (double)v[e].y;
                        part += K * (re * re + im * im);
                    }
                    acc.add(part);
                    break;
                }
                default:
                    break;
            }
        }

        if (a.store) {
            cx<T>* out = reinterpret_cast<cx<T>*>(a.out) + base;
#pragma unroll
            for (int e = 0; e < E; ++e) out[(long)L::index(t, e) * stride] = v[e];
        }
    }

    return acc;
}

// One field: a persistent grid walks the tiles.
// MAXT threads per CTA at most, MINB resident CTAs per SM: the register
// budget per thread is 65536 / (MAXT * MINB) (256 x 2: 128 registers;
// 512 x 2: 64 registers for plans with 8 values per thread).
template <typename T, int N, int RA, int RB, int P, bool STRIDED, bool EXT, int RC = 0,
          int MAXT = kMaxPassThreads, int MINB = 2>
__global__ void __launch_bounds__(MAXT, MINB) k_pass(const PassArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_wait();
    KSum acc =
        pass_tiles<T, N, RA, RB, P, STRIDED, EXT, RC>(a, blockIdx.x, gridDim.x, smem_raw);
    pdl_launch_dependents();
    if (a.red.kind != RED_NONE) {
        __syncthreads();  // smem is reused as reduction scratch
        grid_reduce_finish(acc, reinterpret_cast<double*>(smem_raw), a.red, gridDim.x,
                           blockIdx.x);
    }
}

// Many fields of the same length at once (independent solves): one CTA per
// tile, tile_prefix[s] the first CTA of solve s.  A solve whose *active flag
// is 0 (converged) is skipped; each solve reduces over its own tiles.
template <typename T, int N, int RA, int RB, int P, bool STRIDED, int RC = 0,
          int MAXT = kMaxPassThreads, int MINB = 2>
__global__ void __launch_bounds__(MAXT, MINB)
    k_pass_batch(const PassArgs* __restrict__ args, const long* __restrict__ tile_prefix,
                 int nsolves) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_wait();
    const long b = blockIdx.x;
    int lo = 0, hi = nsolves - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile_prefix[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const PassArgs& a = args[lo];
    if (a.active && *a.active == 0) return;
    const long tile = b - tile_prefix[lo];
    KSum acc = pass_tiles<T, N, RA, RB, P, STRIDED, false, RC>(a, tile, a.ntiles, smem_raw);
    pdl_launch_dependents();
    if (a.red.kind != RED_NONE) {
        __syncthreads();
        grid_reduce_finish(acc, reinterpret_cast<double*>(smem_raw), a.red,
                           (unsigned)a.ntiles, (unsigned)tile);
    }
}

}  // namespace gpue
