// pass.cuh -- one full-field read+write pass over lines of one axis.
//
// A pass loads C lines per CTA (rows for axis 0; C adjacent columns for the
// strided axes 1 and 2, so every row segment is one 32-byte sector for
// complex64), runs a short program of operations on the registers, and stores
// the lines back.  The operations are the pieces of GPUE's split step
// (src/evolution.cu:727-870), fused so each pass touches HBM once:
//
//   OP_SCALE   psi *= pending renormalisation 1/sqrt(sum|psi|^2 dV)
//              (parSum/scalarDiv_wfcNorm, src/split_op.cu:83-129, deferred to
//              the next pass that reads the field)
//   OP_VHALF   psi *= exp(-(V + gN|psi|^2) Dt/(2 hbar))        imaginary time
//              psi *= exp(-i(V + gN|psi|^2) Dt/(2 hbar))       real time
//              (cMultDensity, src/kernels.cu:365-388; linear form cMult)
//   OP_FFT_F / OP_FFT_I   1D DFT along the pass axis, times 1/sqrt(n)
//              (cufftExecZ2Z + scalarMult, src/evolution.cu:758-777)
//   OP_KPHASE  psi *= exp(-K Dt/hbar) / exp(-i K Dt/hbar),
//              K = hbar^2/(2m) |p|^2 (src/operators.cu:460-469, 1081-1103)
//   OP_GAUGE   psi *= exp(-A_a p_a gdt) / exp(-i A_a p_a dt) along the pass
//              axis (apply_gauge, src/evolution.cu:5-257; aux_fields
//              src/operators.cu:1089-1110)
//   OP_NORM    accumulate sum |psi|^2 (FP64, compensated) -> renorm scale
//   OP_EKIN    accumulate sum K |psi_k|^2 (FP64, compensated)
//
// V, K and the imaginary/real-time factors are separable per axis for the
// harmonic trap with the rotation gauge (V = Vx(x) + Vy(y) + Vz(z) including
// m|A|^2/2), so the factors come from small per-axis tables computed in FP64
// on the host (rounded to FP32 for the complex64 form); the nonlinear and
// gauge phases are evaluated per point.

#pragma once

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
    int kind;           // RED_NONE / RED_NORM (writes 1/sqrt(sum dV)) / RED_SUM
    double2* partials;  // [gridDim.x] (sum, compensation)
    unsigned* counter;  // zero between reductions; reset by the last CTA
    double* out;
    double dV;
};

struct PassArgs {
    const void* in;
    void* out;
    int axis;  // 0: x rows (contiguous), 1: y lines (stride nx), 2: z lines
    int nx, ny, nz;
    int nops;
    int ops[kMaxOps];
    int store;   // write the lines back
    int gstate;  // 0 imaginary time, 1 real time
    int gpe;     // nonlinear term on
    double nl_coef;     // gN * (Dt/2) / hbar
    double gauge_coef;  // A_axis = gauge_coef * pos[gauge_src][.]
    int gauge_src;      // axis whose coordinate A_axis depends on
    double gauge_dt;    // gdt * ramp exponent (imaginary) or dt (real)
    double kin_coef;    // hbar^2 / (2 m), for OP_EKIN
    const void* vfac[3];  // cx<T>[n_a]: per-axis V half-step factor
    const void* kfac[3];  // cx<T>[n_a]: per-axis kinetic factor
    const double* pos[3];
    const double* mom[3];
    const void* tw;  // cx<T>[N]: W_N^k for this axis
    double inv_sqrt_n;
    RedArgs red;
    const double* scale_in;  // OP_SCALE factor
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
// needs 2*(blockDim/32) doubles and must not be in use by other threads.
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
// index order (deterministic) and writes the result.  Must be called by all
// threads of the block.
__device__ __forceinline__ void grid_reduce_finish(KSum k, double* scratch, const RedArgs& a) {
    __shared__ unsigned s_last;
    k = block_reduce(k, scratch);
    if (threadIdx.x == 0) {
        a.partials[blockIdx.x] = make_double2(k.s, k.c);
        __threadfence();
        unsigned prev = atomicAdd(a.counter, 1u);
        s_last = (prev == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        KSum t{0.0, 0.0};
        for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
            double2 p = __ldcg(a.partials + i);
            t.merge(p.x, p.y);
        }
        __syncthreads();
        t = block_reduce(t, scratch);
        if (threadIdx.x == 0) {
            double sum = t.s + t.c;
            if (a.kind == RED_NORM)
                a.out[0] = 1.0 / sqrt(sum * a.dV);
            else
                a.out[0] = sum;
            *a.counter = 0u;
        }
    }
}

// ------------------------------------------------------------- helpers --

template <typename T>
__device__ __forceinline__ cx<T> ldc(const void* p, int i) {
    return reinterpret_cast<const cx<T>*>(p)[i];
}

__device__ __forceinline__ void sincos_t(double a, double* s, double* c) { sincos(a, s, c); }
__device__ __forceinline__ void sincos_t(float a, float* s, float* c) { sincosf(a, s, c); }
__device__ __forceinline__ double exp_t(double a) { return exp(a); }
__device__ __forceinline__ float exp_t(float a) { return expf(a); }

// ---------------------------------------------------------------- kernel --

constexpr int kMaxPassThreads = 256;

// C = blockDim.x / P lines per CTA (a launch parameter).
template <typename T, int N, int RA, int RB, int P, bool STRIDED>
__global__ void __launch_bounds__(kMaxPassThreads) k_pass(const PassArgs a) {
    using L = LineFFT<T, N, RA, RB, P>;
    constexpr int E = L::E;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);

    const int C = blockDim.x / P;
    int c, t;
    if constexpr (STRIDED) {
        c = threadIdx.x % C;
        t = threadIdx.x / C;
    } else {
        t = threadIdx.x % P;
        c = threadIdx.x / P;
    }
    T* sre = smem + c * 2 * L::LS;
    T* sim = sre + L::LS;

    const long line = (long)blockIdx.x * C + c;
    const long nxy = (long)a.nx * a.ny;
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

    auto sync = [] {
        if constexpr (STRIDED || P > 32) __syncthreads();
        else __syncwarp();
    };

    const cx<T>* __restrict__ tw = reinterpret_cast<const cx<T>*>(a.tw);
    cx<T> v[E];
    {
        const cx<T>* in = reinterpret_cast<const cx<T>*>(a.in) + base;
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = in[(long)L::index(t, e) * stride];
    }

    KSum acc{0.0, 0.0};
    const T isn = (T)a.inv_sqrt_n;

    for (int o = 0; o < a.nops; ++o) {
        switch (a.ops[o]) {
            case OP_FFT_F: {
                L::template run<false>(v, t, sre, sim, tw, sync);
#pragma unroll
                for (int e = 0; e < E; ++e) v[e] = cscale(v[e], isn);
                break;
            }
            case OP_FFT_I: {
                L::template run<true>(v, t, sre, sim, tw, sync);
#pragma unroll
                for (int e = 0; e < E; ++e) v[e] = cscale(v[e], isn);
                break;
            }
            case OP_SCALE: {
                const T s = (T)(*a.scale_in);
#pragma unroll
                for (int e = 0; e < E; ++e) v[e] = cscale(v[e], s);
                break;
            }
            case OP_VHALF:
            case OP_KPHASE: {
                const void* const* fac = (a.ops[o] == OP_VHALF) ? a.vfac : a.kfac;
                // factor of the two line coordinates
                cx<T> lf;
                if (a.axis == 0) lf = cmul(ldc<T>(fac[1], yi), ldc<T>(fac[2], zi));
                else if (a.axis == 1) lf = cmul(ldc<T>(fac[0], xi), ldc<T>(fac[2], zi));
                else lf = cmul(ldc<T>(fac[0], xi), ldc<T>(fac[1], yi));
                const void* fa = fac[a.axis];
                const bool nl = (a.ops[o] == OP_VHALF) && a.gpe;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    cx<T> f = cmul(ldc<T>(fa, L::index(t, e)), lf);
                    if (nl) {
                        const T gd = (T)a.nl_coef * (v[e].x * v[e].x + v[e].y * v[e].y);
                        if (a.gstate == 0) {
                            f = cscale(f, exp_t(-gd));
                        } else {
                            T s, co;
                            sincos_t(-gd, &s, &co);
                            f = cmul(f, cx<T>{co, s});
                        }
                    }
                    v[e] = cmul(f, v[e]);
                }
                break;
            }
            case OP_GAUGE: {
                const int src = a.gauge_src;
                const int sidx = (src == 0) ? xi : (src == 1) ? yi : zi;
                const double coef = a.gauge_coef * a.pos[src][sidx] * a.gauge_dt;
                const double* mom = a.mom[a.axis];
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const T ang = (T)(coef * mom[L::index(t, e)]);
                    cx<T> f;
                    if (a.gstate == 0) {
                        f = cx<T>{exp_t(-ang), (T)0};
                    } else {
                        T s, co;
                        sincos_t(-ang, &s, &co);
                        f = cx<T>{co, s};
                    }
                    v[e] = cmul(v[e], f);
                }
                break;
            }
            case OP_NORM: {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const double re = (double)v[e].x, im = (double)v[e].y;
                    acc.add(re * re + im * im);
                }
                break;
            }
            case OP_EKIN: {
                const double* m0 = a.mom[0];
                const double* m1 = a.mom[1];
                const double* m2 = a.mom[2];
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int k = L::index(t, e);
                    const double px = m0[a.axis == 0 ? k : xi];
                    const double py = m1[a.axis == 1 ? k : yi];
                    const double pz = m2[a.axis == 2 ? k : zi];
                    const double K = a.kin_coef * (px * px + py * py + pz * pz);
                    const double re = (double)v[e].x, im = (double)v[e].y;
                    acc.add(K * (re * re + im * im));
                }
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

    if (a.red.kind != RED_NONE) {
        __syncthreads();  // smem is reused as reduction scratch
        grid_reduce_finish(acc, reinterpret_cast<double*>(smem_raw), a.red);
    }
}

}  // namespace gpue
