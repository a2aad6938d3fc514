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

template <typename T>
__global__ void __launch_bounds__(256) k_energy_real(const EnergyArgs a) {
    __shared__ double scratch[16];
    const cx<T>* psi = reinterpret_cast<const cx<T>*>(a.psi);
    const double s = a.scale ? *a.scale : 1.0;
    const long nxy = (long)a.nx * a.ny;
    KSum acc{0.0, 0.0};
    for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < a.N;
         g += (long)gridDim.x * blockDim.x) {
        const int xi = (int)(g % a.nx);
        const int yi = (int)((g / a.nx) % a.ny);
        const int zi = (int)(g / nxy);
        const cx<T> pv = psi[g];
        const double px = s * (double)pv.x, py = s * (double)pv.y;
        const double r = px * px + py * py;
        const double V = a.vtab ? a.vtab[g] : a.vreal[0][xi] + a.vreal[1][yi] + a.vreal[2][zi];
        double e = a.gpe ? r * (V + 0.5 * a.gN * r) : r * V;
        if (a.lterm) {
            auto dfwd = [&](long stride, double d, double& ox, double& oy) {
                if (g + stride < a.N) {
                    const cx<T> q = psi[g + stride];
                    ox = (s * (double)q.x - px) / d;
                    oy = (s * (double)q.y - py) / d;
                } else {
                    ox = px / d;
                    oy = py / d;
                }
            };
            double dxr, dxi, dyr, dyi;
            dfwd(1, a.dx, dxr, dxi);
            dfwd(a.nx, a.dy, dyr, dyi);
            const double Ax = a.atab[0] ? a.atab[0][g] : a.ax_coef * a.pos[1][yi];
            const double Ay = a.atab[1] ? a.atab[1][g] : a.ay_coef * a.pos[0][xi];
            double lr = dxr * Ax + dyr * Ay;
            double li = dxi * Ax + dyi * Ay;
            if (a.dim == 3 && a.atab[2]) {
                double dzr, dzi;
                dfwd(nxy, a.dz, dzr, dzi);
                lr += dzr * a.atab[2][g];
                li += dzi * a.atab[2][g];
            }
            // i*hbar*l, then Re[conj(p) * (i hbar l)]
            const double ir = -a.hbar * li, ii = a.hbar * lr;
            e += px * ir + py * ii;
        }
        acc.add(e);
    }
    grid_reduce_finish(acc, scratch, a.red);
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
    grid_reduce_finish(acc, scratch, red);
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
