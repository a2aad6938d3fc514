// aux_kernels.cuh -- elementwise and reduction kernels around the passes.
#pragma once

#include "pass.cuh"

namespace gpue {

// Real-space part of energy_calc (src/split_op.cu:208-375):
//   sum_g |psi|^2 (V + gN|psi|^2/2)                         (gpe)
//   sum_g |psi|^2 V                                         (linear)
// plus, with the gauge on and dim > 1, Re[conj(psi) i hbar (Ax d+x psi +
// Ay d+y psi + Az d+z psi)] where d+ is GPUE's derive() (src/kernels.cu:58-71):
// a forward difference over the flat index with stride 1, nx, nx*ny, and
// psi[g]/d where g+stride runs past the end (no periodic wrap; rows run on
// into the next row).  V = Vx(x)+Vy(y)+Vz(z) and A = (ax_coef*y, ay_coef*x, 0)
// for the rotation gauge.  psi is scaled by *scale when scale != nullptr.
struct EnergyArgs {
    const void* psi;
    long N;
    int nx, ny, nz, dim;
    const double* scale;
    const double* vreal[3];
    const double* pos[3];
    double gN;
    int gpe;
    int lterm;
    double ax_coef, ay_coef;
    double dx, dy, dz;
    double hbar;
    RedArgs red;
    const double* vtab;     // full-field V (parameter-file form), else separable
    const double* atab[3];  // full-field A (parameter-file form), else rotation
};

// GPUE's derive() at flat index g: (psi[g+stride] - psi[g]) / d, or
// psi[g] / d where g+stride runs past the end.  (px, py) = s*psi[g].
template <typename T>
__device__ __forceinline__ void dfwd(const cx<T>* psi, long N, long g, long stride, double s,
                                     double px, double py, double d, double& ox, double& oy) {
    if (g + stride < N) {
        const cx<T> q = psi[g + stride];
        ox = (s * (double)q.x - px) / d;
        oy = (s * (double)q.y - py) / d;
    } else {
        ox = px / d;
        oy = py / d;
    }
}

// Re[conj(psi) i hbar (Ax d+x psi + Ay d+y psi [+ Az d+z psi])] at point g.
template <typename T>
__device__ __forceinline__ double gauge_energy(const EnergyArgs& a, const cx<T>* psi, long g,
                                               int xi, int yi, long nxy, double s, double px,
                                               double py) {
    double dxr, dxi, dyr, dyi;
    dfwd(psi, a.N, g, 1, s, px, py, a.dx, dxr, dxi);
    dfwd(psi, a.N, g, a.nx, s, px, py, a.dy, dyr, dyi);
    const double Ax = a.atab[0] ? a.atab[0][g] : a.ax_coef * a.pos[1][yi];
    const double Ay = a.atab[1] ? a.atab[1][g] : a.ay_coef * a.pos[0][xi];
    double lr = dxr * Ax + dyr * Ay;
    double li = dxi * Ax + dyi * Ay;
    if (a.dim == 3 && a.atab[2]) {
        double dzr, dzi;
        dfwd(psi, a.N, g, nxy, s, px, py, a.dz, dzr, dzi);
        lr += dzr * a.atab[2][g];
        li += dzi * a.atab[2][g];
    }
    // i*hbar*l, then Re[conj(p) * (i hbar l)]
    const double ir = -a.hbar * li, ii = a.hbar * lr;
    return px * ir + py * ii;
}

template <typename T>
__device__ __forceinline__ KSum energy_real_points(const EnergyArgs& a, long g0, long gstep) {
    const cx<T>* psi = reinterpret_cast<const cx<T>*>(a.psi);
    const double s = a.scale ? *a.scale : 1.0;
    const long nxy = (long)a.nx * a.ny;
    KSum acc{0.0, 0.0};
    for (long g = g0; g < a.N; g += gstep) {
        const int xi = (int)(g % a.nx);
        const int yi = (int)((g / a.nx) % a.ny);
        const int zi = (int)(g / nxy);
        const cx<T> pv = psi[g];
        const double px = s * (double)pv.x, py = s * (double)pv.y;
        const double r = px * px + py * py;
        const double V = a.vtab ? a.vtab[g] : a.vreal[0][xi] + a.vreal[1][yi] + a.vreal[2][zi];
        double e = a.gpe ? r * (V + 0.5 * a.gN * r) : r * V;
        if (a.lterm) e += gauge_energy<T>(a, psi, g, xi, yi, nxy, s, px, py);
        acc.add(e);
    }
    return acc;
}

template <typename T>
__global__ void __launch_bounds__(256) k_energy_real(const EnergyArgs a) {
    __shared__ double scratch[16];
    KSum acc = energy_real_points<T>(a, (long)blockIdx.x * blockDim.x + threadIdx.x,
                                     (long)gridDim.x * blockDim.x);
    grid_reduce_finish(acc, scratch, a.red, gridDim.x, blockIdx.x);
}

// Independent solves at once: `per` CTAs per solve, each solve reducing over
// its own CTAs; converged solves (*active == 0) are skipped.
template <typename T>
__global__ void __launch_bounds__(256) k_energy_real_batch(const EnergyArgs* __restrict__ args,
                                                          const int* const* __restrict__ active,
                                                          int per) {
    __shared__ double scratch[16];
    const int s = blockIdx.x / per, b = blockIdx.x % per;
    if (active[s] && *active[s] == 0) return;
    const EnergyArgs& a = args[s];
    KSum acc = energy_real_points<T>(a, (long)b * blockDim.x + threadIdx.x, (long)per * blockDim.x);
    grid_reduce_finish(acc, scratch, a.red, per, b);
}

// Observables of one state (gpue_observables_get): the real-space energy
// terms, trapezoid density moments and <L_z>, reduced in FP64 per quantity.
// Each CTA writes kObsN compensated partials ([q][gridDim.x]); the last CTA to
// arrive sums every quantity in CTA order (deterministic) into out[q].
enum ObsQ {
    kObsNorm, kObsPot, kObsInt, kObsRot, kObsX, kObsY, kObsZ, kObsR2, kObsQ, kObsLz, kObsN
};

struct ObsArgs {
    EnergyArgs e;
    double2* partials;  // [kObsN][gridDim.x]
    unsigned* counter;  // zero between launches; reset by the last CTA
    double* out;        // [kObsN]
    double* ereal;      // optional: potential + interaction + rotation sums (energy_calc's
                        // real-space part, as k_energy_real leaves it)
};

__device__ __forceinline__ double trapz_w(int i, int n) {
    return (n > 1 && (i == 0 || i == n - 1)) ? 0.5 : 1.0;
}

template <typename T>
__global__ void __launch_bounds__(256) k_observables(const ObsArgs o) {
    __shared__ double scratch[kObsN][16];
    __shared__ unsigned s_last;
    const EnergyArgs& a = o.e;
    const cx<T>* psi = reinterpret_cast<const cx<T>*>(a.psi);
    const double s = a.scale ? *a.scale : 1.0;
    const long nxy = (long)a.nx * a.ny;
    KSum acc[kObsN];
#pragma unroll
    for (int q = 0; q < kObsN; ++q) acc[q] = KSum{0.0, 0.0};
    for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < a.N;
         g += (long)gridDim.x * blockDim.x) {
        const int xi = (int)(g % a.nx);
        const int yi = (int)((g / a.nx) % a.ny);
        const int zi = (int)(g / nxy);
        const cx<T> pv = psi[g];
        const double px = s * (double)pv.x, py = s * (double)pv.y;
        const double r = px * px + py * py;
        const double V = a.vtab ? a.vtab[g] : a.vreal[0][xi] + a.vreal[1][yi] + a.vreal[2][zi];
        acc[kObsNorm].add(r);
        acc[kObsPot].add(r * V);
        if (a.gpe) acc[kObsInt].add(0.5 * a.gN * r * r);
        if (a.lterm) acc[kObsRot].add(gauge_energy<T>(a, psi, g, xi, yi, nxy, s, px, py));
        const double X = a.pos[0][xi];
        const double Y = a.dim > 1 ? a.pos[1][yi] : 0.0;
        const double Z = a.dim > 2 ? a.pos[2][zi] : 0.0;
        const double wr = r * trapz_w(xi, a.nx) * trapz_w(yi, a.ny) * trapz_w(zi, a.nz);
        acc[kObsX].add(wr * X);
        acc[kObsY].add(wr * Y);
        acc[kObsZ].add(wr * Z);
        acc[kObsR2].add(wr * (X * X + Y * Y));
        acc[kObsQ].add(wr * (X * X - Y * Y));
        if (a.dim > 1) {
            // -i hbar (x d+y - y d+x) psi, then Re[conj(p) * that]
            double dxr, dxi, dyr, dyi;
            dfwd(psi, a.N, g, 1, s, px, py, a.dx, dxr, dxi);
            dfwd(psi, a.N, g, a.nx, s, px, py, a.dy, dyr, dyi);
            const double Dr = X * dyr - Y * dxr, Di = X * dyi - Y * dxi;
            acc[kObsLz].add(a.hbar * (px * Di - py * Dr));
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < kObsN; ++q) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double os = __shfl_down_sync(0xffffffffu, acc[q].s, off);
            const double oc = __shfl_down_sync(0xffffffffu, acc[q].c, off);
            acc[q].merge(os, oc);
        }
        if (lane == 0) {
            scratch[q][2 * w] = acc[q].s;
            scratch[q][2 * w + 1] = acc[q].c;
        }
    }
    __syncthreads();
    if (threadIdx.x < kObsN) {
        const int q = threadIdx.x;
        KSum t{scratch[q][0], scratch[q][1]};
        for (int i = 1; i < nw; ++i) t.merge(scratch[q][2 * i], scratch[q][2 * i + 1]);
        o.partials[(long)q * gridDim.x + blockIdx.x] = make_double2(t.s, t.c);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(o.counter, 1u);
        s_last = (prev == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    __shared__ double fin[kObsN];
    if (threadIdx.x < kObsN) {
        const int q = threadIdx.x;
        KSum t{0.0, 0.0};
        for (unsigned i = 0; i < gridDim.x; ++i) {
            const double2 p = __ldcg(o.partials + (long)q * gridDim.x + i);
            t.merge(p.x, p.y);
        }
        fin[q] = t.s + t.c;
        o.out[q] = fin[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (o.ereal) *o.ereal = fin[kObsPot] + fin[kObsInt] + fin[kObsRot];
        *o.counter = 0u;
    }
}

// Energy check of batched solves, one block.  flags[2] counts a solve's
// checks; check k (from 0) is taken after step k*every + step_base - 1, so
// with step_base 1 the checks fall on evolve's i % energy_calc_steps == 0
// steps (src/evolution.cu:872-905) and a solve that stops there has run
// k*every + step_base steps.  E = (ekin/N + ereal) dV; from the second check
// on, an imaginary-time solve whose |E_previous - E| < threshold (absolute,
// or times E_previous) is marked done.  *nactive receives the number of
// solves still running.
struct CheckArgs {
    double* scal;       // the solve's scalar slots
    int* flags;         // [0] active, [1] steps done when it stopped, [2] checks
    double inv_n;       // 1/N
    double dV;
    int slot_ekin, slot_ereal, slot_eold, slot_e;
};

static __global__ void k_batch_check(const CheckArgs* __restrict__ args, int n, int every,
                              int step_base, double thr, int thr_abs, int can_stop,
                              int* nactive) {
    __shared__ int running;
    if (threadIdx.x == 0) running = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        const CheckArgs& c = args[s];
        if (c.flags[0] == 0) continue;
        const int k = c.flags[2];
        const double E = (c.scal[c.slot_ekin] * c.inv_n + c.scal[c.slot_ereal]) * c.dV;
        const double old = c.scal[c.slot_eold];
        const bool stop = thr_abs ? fabs(old - E) < thr : fabs(old - E) < thr * old;
        if (can_stop && k > 0 && stop) {
            c.flags[0] = 0;
            c.flags[1] = k * every + step_base;
        } else {
            atomicAdd(&running, 1);
        }
        c.flags[2] = k + 1;
        c.scal[c.slot_eold] = E;
        c.scal[c.slot_e] = E;
    }
    __syncthreads();
    if (threadIdx.x == 0) *nactive = running;
}

// One record per batched solve, gathered for a single device-to-host copy.
struct BatchOut {
    double energy;
    int active;
    int steps;
    int checks;
    int pad;
};

static __global__ void k_batch_gather(const CheckArgs* __restrict__ args, int n, BatchOut* out) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const CheckArgs& c = args[s];
        out[s].energy = c.scal[c.slot_e];
        out[s].active = c.flags[0];
        out[s].steps = c.flags[1];
        out[s].checks = c.flags[2];
        out[s].pad = 0;
    }
}

// sum |psi|^2 (optionally times *scale^2) -> RED_SUM/RED_NORM
template <typename T>
__global__ void __launch_bounds__(256) k_norm(const void* psi_, long N, RedArgs red) {
    __shared__ double scratch[16];
    const cx<T>* psi = reinterpret_cast<const cx<T>*>(psi_);
    KSum acc{0.0, 0.0};
    for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < N;
         g += (long)gridDim.x * blockDim.x) {
        const cx<T> v = psi[g];
        acc.add((double)v.x * v.x + (double)v.y * v.y);
    }
    grid_reduce_finish(acc, scratch, red, gridDim.x, blockIdx.x);
}

template <typename T>
__global__ void k_scale(void* psi_, long N, const double* scale) {
    cx<T>* psi = reinterpret_cast<cx<T>*>(psi_);
    const T s = (T)*scale;
    for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < N;
         g += (long)gridDim.x * blockDim.x)
        psi[g] = cscale(psi[g], s);
}

template <typename TI, typename TO>
__global__ void k_convert(const void* in_, void* out_, long N) {
    const cx<TI>* in = reinterpret_cast<const cx<TI>*>(in_);
    cx<TO>* out = reinterpret_cast<cx<TO>*>(out_);
    for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < N;
         g += (long)gridDim.x * blockDim.x)
        out[g] = cx<TO>{(TO)in[g].x, (TO)in[g].y};
}

}  // namespace gpue
