// gpe_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A CPU, FP64 restatement of GPUE's split-operator Gross-Pitaevskii step.  It
// is the checker for the CUDA path and the timed CPU baseline; the product
// library never imports, links or calls it.  It follows the reference's data
// flow literally: real operator tables (V, K, A) are built the way
// operators.cu builds them, turned into the imaginary/real-time operators the
// way aux_fields does, and applied in evolve()'s order with an unnormalised
// DFT followed by 1/sqrt(n) scaling, as GPUE does with cuFFT.
//
// Reference (GPUE-group/GPUE) lines restated here:
//   step order               src/evolution.cu:727-870
//   gauge passes, flip order src/evolution.cu:5-160 (3D), 163-257 (2D)
//   ramp exponent            src/evolution.cu:409-427, kernels.cu:491-497
//   nonlinear half step      src/kernels.cu:365-388  (cMultDensity)
//   AST step kernels         src/kernels.cu:165-187, 391-422, 632-665
//   grids                    src/operators.cu:277-432, src/init.cu:120-170
//   K, A, V, initial wfc     src/operators.cu:460-469, 621-647, 994-1008, 1031-1050
//   operator tables          src/operators.cu:1069-1111 (aux_fields)
//   renormalisation          src/split_op.cu:83-129
//   energy                   src/split_op.cu:208-375, derive src/kernels.cu:58-71
//   AST evaluation           src/dynamic.cu:527-603
//   2D vortex finder         src/tracker.cu:102-166 (Tracker::findVortex)
//
// The DFT is this file's own mixed-radix Stockham transform (radices 2,3,4,5
// and a direct DFT for other primes); FFTW is not available.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

namespace {

// ---------------------------------------------------------------- FFT ----

struct Plan {
    int n = 0;
    std::vector<int> radices;
    std::vector<cd> w;  // w[k] = exp(-2 pi i k / n)
};

std::mutex g_plan_mu;
std::map<int, Plan*> g_plans;

const Plan* get_plan(int n) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find(n);
    if (it != g_plans.end()) return it->second;
    Plan* p = new Plan;
    p->n = n;
    int m = n;
    while (m % 4 == 0) { p->radices.push_back(4); m /= 4; }
    while (m % 2 == 0) { p->radices.push_back(2); m /= 2; }
    for (int f = 3; m > 1; f += 2) {
        while (m % f == 0) { p->radices.push_back(f); m /= f; }
    }
    p->w.resize(n);
    const long double tau = 6.283185307179586476925286766559L;
    for (int k = 0; k < n; ++k) {
        long double a = -tau * (long double)k / (long double)n;
        p->w[k] = cd((double)cosl(a), (double)sinl(a));
    }
    g_plans[n] = p;
    return p;
}

// Unnormalised DFT of one contiguous line (sign -1 forward, +1 inverse),
// Stockham autosort; work must hold n elements.
void fft_line(const Plan* p, cd* x, cd* work, int sign) {
    const int n = p->n;
    if (n == 1) return;
    cd* in = x;
    cd* out = work;
    int Ns = 1;
    cd v[64];
    for (int R : p->radices) {
        const int m = n / R;
        const int tstep = n / (Ns * R);
        for (int j = 0; j < m; ++j) {
            const int jm = j % Ns;
            for (int r = 0; r < R; ++r) {
                cd a = in[j + r * m];
                if (r && jm) {
                    cd t = p->w[(jm * r * tstep) % n];
                    if (sign > 0) t = std::conj(t);
                    a *= t;
                }
                v[r] = a;
            }
            const int base = (j / Ns) * Ns * R + jm;
            if (R == 2) {
                out[base] = v[0] + v[1];
                out[base + Ns] = v[0] - v[1];
            } else if (R == 4) {
                cd s02 = v[0] + v[2], d02 = v[0] - v[2];
                cd s13 = v[1] + v[3], d13 = v[1] - v[3];
                // multiply d13 by -i (forward) or +i (inverse)
                cd jd13 = (sign < 0) ? cd(d13.imag(), -d13.real())
                                     : cd(-d13.imag(), d13.real());
                out[base] = s02 + s13;
                out[base + Ns] = d02 + jd13;
                out[base + 2 * Ns] = s02 - s13;
                out[base + 3 * Ns] = d02 - jd13;
            } else {
                const int step = n / R;
                for (int k = 0; k < R; ++k) {
                    cd acc = v[0];
                    for (int r = 1; r < R; ++r) {
                        cd t = p->w[((r * k) % R) * step];
                        if (sign > 0) t = std::conj(t);
                        acc += v[r] * t;
                    }
                    out[base + k * Ns] = acc;
                }
            }
        }
        Ns *= R;
        std::swap(in, out);
    }
    if (in != x) std::memcpy(x, in, sizeof(cd) * n);
}

// Transform `lines` lines of length n, element stride `stride`, line starts
// given by line_off(l).  Lines are gathered into a contiguous buffer.
template <typename F>
void fft_lines(cd* data, int n, long stride, long lines, F line_off, int sign,
               double scale) {
    const Plan* p = get_plan(n);
#pragma omp parallel
    {
        std::vector<cd> buf(n), work(n);
#pragma omp for schedule(static)
        for (long l = 0; l < lines; ++l) {
            cd* base = data + line_off(l);
            for (int i = 0; i < n; ++i) buf[i] = base[i * stride];
            fft_line(p, buf.data(), work.data(), sign);
            for (int i = 0; i < n; ++i) base[i * stride] = buf[i] * scale;
        }
    }
}

// ------------------------------------------------------------ AST eval ---

}  // namespace

extern "C" {

// Node layout of GPUE's EqnNode_gpu (include/ds.h:71-80): a flattened tree,
// root at index 0, children by index, leaves either a constant or one of the
// variables x, y, z, t.
typedef struct {
    double val;
    int32_t is_dynamic;
    int32_t var;  // 'x','y','z','t'
    int32_t left, right;
    int32_t op_num;
} orc_node;

}  // extern "C"

namespace {

double factorial_d(double val) {
    double ret = val;
    if (val < 1) return 1;
    for (int i = (int)std::floor(val) - 1; i > 0; --i) ret *= i;
    return ret;
}

cd cpow_int(cd a, int b) {  // src/kernels.cu:12-16
    double r = std::sqrt(a.real() * a.real() + a.imag() * a.imag());
    double th = std::atan(a.imag() / a.real());
    return cd(std::pow(r, b) * std::cos(b * th), std::pow(r, b) * std::sin(b * th));
}

cd poly_i(int v, cd x, int n) {  // src/dynamic.cu:116-127
    cd ival(0, 0);
    x = cd(0, 1) * x;
    for (int i = 0; i < n; ++i) {
        double b = std::pow(-1.0, i) * (factorial_d(n + i - 1) * std::pow((double)n, 1 - 2 * i)) /
                   (factorial_d(i) * factorial_d(n - i) * factorial_d(v + i));
        cd s = cpow_int(x * 0.5, 2 * i + v) * b;
        ival += s;
    }
    return ival;
}

double k2n_eval(double a, double b) {  // src/dynamic.cu:129-141
    cd x(b, 0);
    int n = 30, v = (int)a;
    cd val = (poly_i(-v, x, n) - poly_i(v, x, n)) * (M_PI / (2 * std::sin(n * M_PI)));
    return (val * val).real();
}

double ast_eval(const orc_node* e, double x, double y, double z, double t, int k) {
    const orc_node& nd = e[k];
    if (nd.right < 0 && nd.left < 0) {
        if (nd.is_dynamic) {
            if (nd.var == 'x') return x;
            if (nd.var == 'y') return y;
            if (nd.var == 'z') return z;
            if (nd.var == 't') return t;
        } else {
            return nd.val;
        }
    }
    double a = nd.left > 0 ? ast_eval(e, x, y, z, t, nd.left) : 0.0;
    double b = nd.right > 0 ? ast_eval(e, x, y, z, t, nd.right) : 0.0;
    switch (nd.op_num) {
        case 1: return a + b;
        case 2: return a - b;
        case 3: return a * b;
        case 4: return a / b;
        case 5: return std::pow(a, (int)b);
        case 6: return std::cos(a);
        case 7: return std::sin(a);
        case 8: return std::tan(a);
        case 9: return std::sqrt(a);
        case 10: return std::exp(a);
        case 11: return ((int)a == 0) ? j0(b) : ((int)a == 1) ? j1(b) : jn((int)a, b);
        case 12: return ((int)a == 0) ? y0(b) : ((int)a == 1) ? y1(b) : yn((int)a, b);
        case 13: return k2n_eval(a, b);
    }
    return 0.0;
}

// make_complex (src/kernels.cu:165-187)
inline cd make_complex(double in, int type) {
    if (type == 0) return cd(in, 0);
    if (type == 1) return cd(std::exp(-in), 0);
    return cd(std::cos(-in), std::sin(-in));
}

}  // namespace

extern "C" {

typedef struct {
    int32_t dimnum;           // 2 or 3 (1 accepted)
    int32_t nx, ny, nz;
    double dx, dy, dz;
    double hbar;
    double gN;                // interaction * gDenConst
    double gdt, dt;
    int32_t gpe;              // nonlinear term on (-s)
    int32_t corotating;       // gauge passes and L energy term on (-l)
    int32_t ramp, ramp_type;  // -R
    double omega;             // -w, used by the ramp exponent
    int32_t threads;          // OpenMP threads, 0 = runtime default
    int32_t energy_every;     // energy_calc_steps; 0 = no energy checks
    double threshold;         // early-stop threshold
    int32_t threshold_abs;    // 0: |dE| < thr*E_old (GPUE), 1: |dE| < thr
    // time-dependent AST programs (NULL = use the static tables); positions
    // are (i*dx, j*dy, k*dz) and time = Dt*step, as evolve() passes them
    const orc_node* ast_V;
    const orc_node* ast_K;
    const orc_node* ast_Ax;
    const orc_node* ast_Ay;
    const orc_node* ast_Az;
} orc_cfg;

typedef struct {
    int32_t steps_done;
    int32_t early_stop;
    int32_t n_energies;
    double energy;
} orc_result;

int orc_version(void) { return 1; }

double orc_ast_eval(const orc_node* e, double x, double y, double z, double t) {
    return ast_eval(e, x, y, z, t, 0);
}

// Unnormalised 1D DFT of `howmany` lines (sign -1 forward / +1 inverse).
void orc_fft1d(double* data, int n, int howmany, long stride, long dist, int sign) {
    cd* d = reinterpret_cast<cd*>(data);
    fft_lines(d, n, stride, howmany, [&](long l) { return l * dist; }, sign, 1.0);
}

// generate_p_space (src/operators.cu:336-343) for one axis: x and p grids.
void orc_axis_grid(int n, double xMax, double* x, double* px) {
    const double PI = 3.141592653589793;
    double dx = xMax / (n >> 1);
    double dpx = PI / xMax;
    double pxMax = (PI / xMax) * (n >> 1);
    for (int i = 0; i < n / 2; ++i) {
        x[i] = -xMax + i * dx;
        x[i + n / 2] = i * dx;
        px[i] = i * dpx;
        px[i + n / 2] = -pxMax + i * dpx;
    }
}

// Real operator fields as generate_fields builds them for the harmonic trap
// and the "rotation" gauge (kharmonic_V, simple_K, krotation_Ax/Ay,
// kconstant_A).  items: xMax..a0z as operators.cu:756-795 lays them out is
// not needed; the harmonic V uses omega{X,Y,Z}, gammaY, shifts and mass.
void orc_fields(int dimnum, int nx, int ny, int nz, const double* x, const double* y,
                const double* z, const double* px, const double* py, const double* pz,
                double hbar, double mass, double omegaX, double omegaY, double omegaZ,
                double gammaY, double x0, double y0, double z0, double omega, int rotation,
                double* V, double* K, double* Ax, double* Ay, double* Az) {
    double wz = (dimnum == 3) ? omegaZ : 0.0;  // items[5] is 0 in 2D
    double z0s = (dimnum == 3) ? z0 : 0.0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long g = i + (long)nx * (j + (long)ny * k);
                double ax = 0, ay = 0, az = 0;
                if (rotation) {
                    ax = -y[j] * omega * omegaX;
                    ay = x[i] * omega * omegaY;
                }
                Ax[g] = ax;
                Ay[g] = ay;
                Az[g] = az;
                double vx = omegaX * (x[i] + x0);
                double vy = gammaY * omegaY * (y[j] + y0);
                double vz = 1.0 * wz * (z[k] + z0s);
                V[g] = 0.5 * mass * ((vx * vx + vy * vy + vz * vz) + (ax * ax + ay * ay + az * az));
                K[g] = (hbar * hbar / (2 * mass)) * (px[i] * px[i] + py[j] * py[j] + pz[k] * pz[k]);
            }
}

}  // extern "C"

namespace {

struct Field {
    const orc_cfg* c;
    long N;
    int nx, ny, nz;
    double dV;
};

void fft_nd(const Field& f, cd* psi, int sign) {
    // every axis of the (square/cubic) grid, unnormalised, then 1/sqrt(N)
    const int nx = f.nx, ny = f.ny, nz = f.nz;
    fft_lines(psi, nx, 1, (long)ny * nz, [&](long l) { return l * nx; }, sign, 1.0);
    if (f.c->dimnum > 1)
        fft_lines(psi, ny, nx, (long)nx * nz,
                  [&](long l) { return (l % nx) + (l / nx) * (long)nx * ny; }, sign, 1.0);
    if (f.c->dimnum > 2)
        fft_lines(psi, nz, (long)nx * ny, (long)nx * ny, [&](long l) { return l; }, sign, 1.0);
    double s = 1.0 / std::pow((double)f.N, 0.5);
#pragma omp parallel for schedule(static)
    for (long g = 0; g < f.N; ++g) psi[g] *= s;
}

// 1D transform along one axis, followed by 1/sqrt(n_axis)
void fft_axis(const Field& f, cd* psi, int axis, int sign) {
    const int nx = f.nx, ny = f.ny, nz = f.nz;
    if (axis == 0) {
        fft_lines(psi, nx, 1, (long)ny * nz, [&](long l) { return l * nx; }, sign,
                  1.0 / std::pow((double)nx, 0.5));
    } else if (axis == 1) {
        fft_lines(psi, ny, nx, (long)nx * nz,
                  [&](long l) { return (l % nx) + (l / nx) * (long)nx * ny; }, sign,
                  1.0 / std::pow((double)ny, 0.5));
    } else {
        fft_lines(psi, nz, (long)nx * ny, (long)nx * ny, [&](long l) { return l; }, sign,
                  1.0 / std::pow((double)nz, 0.5));
    }
}

struct Tables {
    const double *V, *K, *Ax, *Ay, *Az, *px, *py, *pz;
};

double energy_impl(const Field& f, const Tables& t, const cd* psi) {
    const orc_cfg* c = f.c;
    const long N = f.N;
    const int nx = f.nx, ny = f.ny;
    std::vector<cd> wk(psi, psi + N);
    fft_nd(f, wk.data(), -1);
#pragma omp parallel for schedule(static)
    for (long g = 0; g < N; ++g) wk[g] *= t.K[g];
    fft_nd(f, wk.data(), +1);
    double sum = 0.0, comp = 0.0;
    // Neumaier-compensated sum of the per-point energy density
    std::vector<double> dens(N);
#pragma omp parallel for schedule(static)
    for (long g = 0; g < N; ++g) {
        cd p = psi[g];
        cd pc = std::conj(p);
        double ek = (pc * wk[g]).real();
        double r = std::norm(p);
        double er;
        if (c->gpe)
            er = (pc * (p * (r * 0.5 * c->gN + t.V[g]))).real();
        else
            er = (pc * (p * t.V[g])).real();
        double e = er + ek;
        if (c->corotating && c->dimnum > 1) {
            auto der = [&](long stride, double d) -> cd {
                if (g + stride < N) return (psi[g + stride] - psi[g]) / d;
                return psi[g] / d;
            };
            cd l = der(1, c->dx) * t.Ax[g];
            l += der(nx, c->dy) * t.Ay[g];
            if (c->dimnum == 3) l += der((long)nx * ny, c->dz) * t.Az[g];
            l *= cd(0, c->hbar);
            e += (pc * l).real();
        }
        dens[g] = e;
    }
    for (long g = 0; g < N; ++g) {
        double y = dens[g];
        double tsum = sum + y;
        if (std::fabs(sum) >= std::fabs(y))
            comp += (sum - tsum) + y;
        else
            comp += (y - tsum) + sum;
        sum = tsum;
    }
    return (sum + comp) * f.dV;
}

}  // namespace

extern "C" {

double orc_energy(const orc_cfg* c, const double* V, const double* K, const double* Ax,
                  const double* Ay, const double* Az, const double* psi_in) {
#ifdef _OPENMP
    if (c->threads > 0) omp_set_num_threads(c->threads);
#endif
    Field f{c, (long)c->nx * c->ny * c->nz, c->nx, c->ny, c->nz, 0};
    f.dV = c->dx;
    if (c->dimnum > 1) f.dV *= c->dy;
    if (c->dimnum > 2) f.dV *= c->dz;
    Tables t{V, K, Ax, Ay, Az, nullptr, nullptr, nullptr};
    return energy_impl(f, t, reinterpret_cast<const cd*>(psi_in));
}

// evolve() (src/evolution.cu:260-908) without I/O and vortex hooks.
// psi: interleaved complex128, x fastest.  energies: optional output of every
// energy computed (capacity nsteps/energy_every + 1).
int orc_evolve(const orc_cfg* c, const double* V, const double* K, const double* Ax,
               const double* Ay, const double* Az, const double* px, const double* py,
               const double* pz, double* psi_io, int nsteps, int gstate, double* energies,
               orc_result* res) {
#ifdef _OPENMP
    if (c->threads > 0) omp_set_num_threads(c->threads);
#endif
    cd* psi = reinterpret_cast<cd*>(psi_io);
    Field f{c, (long)c->nx * c->ny * c->nz, c->nx, c->ny, c->nz, 0};
    f.dV = c->dx;
    if (c->dimnum > 1) f.dV *= c->dy;
    if (c->dimnum > 2) f.dV *= c->dz;
    const long N = f.N;
    const int nx = c->nx, ny = c->ny;
    const double hbar = c->hbar;
    const double Dt = (gstate == 0) ? c->gdt : c->dt;
    Tables t{V, K, Ax, Ay, Az, px, py, pz};

    // operator tables: aux_fields (src/operators.cu:1069-1111)
    std::vector<cd> Vop(N), Kop(N), pAop[3];
    for (int a = 0; a < 3; ++a) pAop[a].resize(N);
#pragma omp parallel for schedule(static)
    for (long g = 0; g < N; ++g) {
        int i = (int)(g % nx), j = (int)((g / nx) % ny), k = (int)(g / ((long)nx * ny));
        double pA[3] = {Ax[g] * px[i], Ay[g] * py[j], Az[g] * pz[k]};
        if (gstate == 0) {
            Vop[g] = cd(std::exp(-V[g] * (c->gdt / (2 * hbar))), 0.0);
            Kop[g] = cd(std::exp(-K[g] * (c->gdt / hbar)), 0.0);
            for (int a = 0; a < 3; ++a) pAop[a][g] = cd(std::exp(-pA[a] * c->gdt), 0);
        } else {
            Vop[g] = cd(std::cos(-V[g] * (c->dt / (2 * hbar))), std::sin(-V[g] * (c->dt / (2 * hbar))));
            Kop[g] = cd(std::cos(-K[g] * (c->dt / hbar)), std::sin(-K[g] * (c->dt / hbar)));
            for (int a = 0; a < 3; ++a)
                pAop[a][g] = cd(std::cos(-pA[a] * c->dt), std::sin(-pA[a] * c->dt));
        }
    }

    auto pos = [&](long g, double& x, double& y, double& z) {
        int i = (int)(g % nx), j = (int)((g / nx) % ny), k = (int)(g / ((long)nx * ny));
        x = i * c->dx;
        y = j * (c->dimnum > 1 ? c->dy : 1.0);
        z = k * (c->dimnum > 2 ? c->dz : 1.0);
    };

    auto half_v = [&](double time) {
#pragma omp parallel for schedule(static)
        for (long g = 0; g < N; ++g) {
            cd p = psi[g];
            if (c->gpe) {
                double gD = c->gN * std::norm(p) * ((0.5 * Dt) / hbar);
                cd val = Vop[g];
                if (c->ast_V) {
                    double x, y, z;
                    pos(g, x, y, z);
                    val = make_complex(ast_eval(c->ast_V, x, y, z, time, 0), gstate + 1);
                }
                if (gstate == 0) {
                    double tmp = val.real() * std::exp(-gD);
                    psi[g] = cd(tmp * p.real() - val.imag() * p.imag(),
                                tmp * p.imag() + val.imag() * p.real());
                } else {
                    cd tmp(val.real() * std::cos(-gD) - val.imag() * std::sin(-gD),
                           val.imag() * std::cos(-gD) + val.real() * std::sin(-gD));
                    psi[g] = tmp * p;
                }
            } else {
                if (c->ast_V) {
                    double x, y, z;
                    pos(g, x, y, z);
                    psi[g] = p * make_complex(ast_eval(c->ast_V, x, y, z, time, 0) * Dt, gstate + 1);
                } else {
                    psi[g] = Vop[g] * p;
                }
            }
        }
    };

    auto gauge_axis = [&](int axis, double time, double rexp) {
        const orc_node* ast = axis == 0 ? c->ast_Ax : axis == 1 ? c->ast_Ay : c->ast_Az;
        fft_axis(f, psi, axis, -1);
#pragma omp parallel for schedule(static)
        for (long g = 0; g < N; ++g) {
            if (ast) {
                double x, y, z;
                pos(g, x, y, z);
                psi[g] *= ast_eval(ast, x, y, z, time, 0);
            } else {
                cd op = pAop[axis][g];
                if (rexp != 1.0) op = cd(std::pow(op.real(), rexp), std::pow(op.imag(), rexp));
                psi[g] = psi[g] * op;
            }
        }
        fft_axis(f, psi, axis, +1);
    };

    double rexp = 1.0;  // cumulative scalarPow exponent under the ramp
    int n_en = 0;
    double old_energy = 0.0, energy = NAN;
    int steps = 0, early = 0;
    for (int i = 0; i < nsteps; ++i) {
        double time = Dt * i;
        if (c->ramp) {
            double w0;
            if (c->ramp_type == 1) w0 = (i == 0) ? c->omega : (double)i / (double)(i + 1);
            else w0 = (i == 0) ? c->omega / (double)nsteps : (double)(i + 1) / (double)i;
            rexp *= w0;
        }
        half_v(time);
        fft_nd(f, psi, -1);
        if (c->ast_K) {
#pragma omp parallel for schedule(static)
            for (long g = 0; g < N; ++g) {
                double x, y, z;
                pos(g, x, y, z);
                psi[g] *= make_complex(ast_eval(c->ast_K, x, y, z, time, 0) * Dt, gstate + 1);
            }
        } else {
#pragma omp parallel for schedule(static)
            for (long g = 0; g < N; ++g) psi[g] = Kop[g] * psi[g];
        }
        fft_nd(f, psi, +1);
        half_v(time);
        if (c->corotating) {
            bool flip = (i % 2) != 0;
            double re = c->ramp ? rexp : 1.0;
            if (c->dimnum == 3) {
                if (flip) { gauge_axis(0, time, re); gauge_axis(1, time, re); gauge_axis(2, time, re); }
                else      { gauge_axis(2, time, re); gauge_axis(1, time, re); gauge_axis(0, time, re); }
            } else if (c->dimnum == 2) {
                if (flip) { gauge_axis(0, time, re); gauge_axis(1, time, re); }
                else      { gauge_axis(1, time, re); gauge_axis(0, time, re); }
            } else {
                gauge_axis(0, time, re);
            }
        }
        if (gstate == 0) {
            double s = 0.0, comp = 0.0;
            for (long g = 0; g < N; ++g) {
                double y = std::norm(psi[g]);
                double ts = s + y;
                comp += (s >= y) ? (s - ts) + y : (y - ts) + s;
                s = ts;
            }
            double norm = std::sqrt((s + comp) * f.dV);
#pragma omp parallel for schedule(static)
            for (long g = 0; g < N; ++g) psi[g] /= norm;
        }
        steps = i + 1;
        if (c->energy_every > 0 && i % c->energy_every == 0) {
            energy = energy_impl(f, t, psi);
            if (energies) energies[n_en] = energy;
            n_en++;
            bool stop;
            if (c->threshold_abs)
                stop = std::fabs(old_energy - energy) < c->threshold;
            else
                stop = std::fabs(old_energy - energy) < c->threshold * old_energy;
            if (i != 0 && stop && gstate == 0) {
                early = 1;
                break;
            }
            old_energy = energy;
        }
    }
    if (res) {
        res->steps_done = steps;
        res->early_stop = early;
        res->n_energies = n_en;
        res->energy = energy;
    }
    return 0;
}

// Standard initial state kstd_wfc (src/operators.cu:1031-1050) before the
// host-side normalisation; phi = -fmod(winding*atan2(y,x), 2pi).
void orc_std_wfc(int nx, int ny, int nz, const double* x, const double* y, const double* z,
                 double Rxy, double a0x, double a0y, double a0z, double winding,
                 double* psi_out) {
    const double PI = 3.141592653589793;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long g = i + (long)nx * (j + (long)ny * k);
                double phi = -std::fmod(winding * std::atan2(y[j], x[i]), 2 * PI);
                double e = std::exp(-(x[i] * x[i] / (Rxy * Rxy * a0x * a0x) +
                                      y[j] * y[j] / (Rxy * Rxy * a0y * a0y) +
                                      z[k] * z[k] / (Rxy * Rxy * a0z * a0z)));
                psi_out[2 * g] = e * std::cos(phi);
                psi_out[2 * g + 1] = -e * std::sin(phi);
            }
}

}  // extern "C"

// ------------------------------------------------------------ vortices --
//
// Tracker::findVortex (src/tracker.cu:102-166), restated.  The plaquettes
// (i, j), i < n-1 the slow (row) index and j < n-1 the contiguous one, are
// visited row by row; those with sqrt(x[i]^2 + x[j]^2) < radius (the x array
// serves both axes: GPUE's grids are square) sum the wrapped phase steps
// arg(w_a) - arg(w_b) around (i,j) -> (i+1,j) -> (i+1,j+1) -> (i,j+1) -> (i,j),
// each phase taken of (w_a conj(w_b)) / |w_b|^2 * |w_b|/|w_a| with atan2 and
// moved from (-inf, -pi] up by 2 pi.  A sum >= 1.9 pi or <= -1.9 pi marks the
// plaquette with |lround(sum / 2 pi)| (findVortex stores -lround for negative
// sums) unless the previous in-radius plaquette in visiting order was marked:
// the two counters findVortex sets to 2 on a mark and decrements after every
// in-radius plaquette skip exactly the next one.  marker (n*n ints) must be
// zero on entry; winding, if not null, receives the signed lround at marked
// plaquettes.  Returns the number of marks.
namespace {
struct c2 {
    double x, y;
};
c2 cdiv_scaled(c2 a, c2 b) {
    // complexScale(complexDiv(a, b), |b| / |a|) (src/minions.cu:62-93)
    const c2 cb{b.x, -b.y};
    const c2 m{a.x * cb.x - a.y * cb.y, a.x * cb.y + a.y * cb.x};
    const double inv = 1.0 / (b.x * b.x + b.y * b.y);
    const c2 q{m.x * inv, m.y * inv};
    const double r = std::sqrt(b.x * b.x + b.y * b.y) / std::sqrt(a.x * a.x + a.y * a.y);
    return c2{q.x * r, q.y * r};
}
}  // namespace

extern "C" int orc_find_vortex(const double* wfc, int n, const double* x, double radius,
                               int* marker, int* winding) {
    const double PI = 3.141592653589793;
    const c2* w = reinterpret_cast<const c2*>(wfc);
    int found = 0;
    bool skip_next = false;  // the previous in-radius plaquette was marked
    for (int i = 0; i < n - 1; ++i) {
        for (int j = 0; j < n - 1; ++j) {
            if (!(std::sqrt(x[i] * x[i] + x[j] * x[j]) < radius)) continue;
            const c2 corner[4] = {w[i * n + j], w[(i + 1) * n + j], w[(i + 1) * n + j + 1],
                                  w[i * n + j + 1]};
            double d[4];
            for (int k = 0; k < 4; ++k) {
                const c2 g = cdiv_scaled(corner[k], corner[(k + 1) & 3]);
                d[k] = std::atan2(g.y, g.x);
                if (d[k] <= -PI) d[k] += 2 * PI;
            }
            const double sum = d[0] + d[1] + d[2] + d[3];
            const bool mark = !skip_next && (sum >= 1.9 * PI || sum <= -1.9 * PI);
            if (mark) {
                const long r = std::lround(sum / (2 * PI));
                marker[i * n + j] = (int)(r < 0 ? -r : r);
                if (winding) winding[i * n + j] = (int)r;
                ++found;
            }
            skip_next = mark;
        }
    }
    return found;
}

