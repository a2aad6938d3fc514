// engine.cu -- host side of the split-operator step behind include/gpue_b200.h.
//
// A context owns the resident wavefunction, per-axis operator tables, the
// FP64 reduction scratch and one CUDA stream.  gpue_evolve() turns each time
// step of GPUE's evolve() (src/evolution.cu:407-904) into a short list of
// fused line passes (pass.cuh), fuses adjacent passes along the same axis
// across step boundaries, and replays the result as captured CUDA graphs in
// segments between energy checks.
//
// Step schedule (R = row pass along x, C = strided pass along y, Z along z;
// flip = i % 2 as GPUE alternates the gauge order):
//   2D          R[scale? V/2 F]  C[F K I]  R[I V/2]                 (+norm)
//   2D gauge 1  R[scale? V/2 F]  C[F K I]  R[I V/2 F Gx I]  C[F Gy I] (+norm)
//   2D gauge 0  R[scale? V/2 F]  C[F K I]  R[I V/2]  C[F Gy I]  R[F Gx I] (+norm)
//   3D          X[scale? V/2 F]  Y[F]  Z[F K I]  Y[I]  X[I V/2] (+gauge passes)
// In real time the last pass of a step and the first pass of the next are
// fused when they share an axis (no renormalisation lies between them).

#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gpue_b200.h"
#include "aux_kernels.cuh"
#include "registry.h"

using namespace gpue;

namespace {

const double kPI = 3.141592653589793;  // GPUE's PI (include/constants.h)

struct Axis {
    int n = 1;
    double xmax = 0, dx = 1;
    std::vector<double> x, p;  // positions, momenta (generate_p_space order)
};

// Device tables for one precision.
struct Tables {
    void* buf = nullptr;
    const void* vfac[3] = {};
    const void* kfac[3] = {};
    const void* tw[3] = {};
    const double* pos[3] = {};
    const double* mom[3] = {};
    const double* vreal[3] = {};
    int built_for = -1;  // gstate of vfac/kfac
};

struct GraphKey {
    int gstate, parity, nsteps, scale_first, energy_last;
    bool operator<(const GraphKey& o) const {
        return std::memcmp(this, &o, sizeof(GraphKey)) < 0;
    }
};

struct Segment {
    cudaGraphExec_t exec = nullptr;
    long launches = 0;
};

}  // namespace

struct gpue_ctx {
    gpue_params p{};
    int dim = 2;
    int prec = GPUE_PREC_FP64;
    Axis ax[3];
    long N = 0;
    double dV = 1;
    int device = 0;
    cudaStream_t stream = nullptr;
    void* psi = nullptr;      // resident state in the context precision
    void* scratch = nullptr;  // N * 16 bytes
    double* scal = nullptr;   // device scalars
    double2* partials = nullptr;
    long partials_cap = 0;
    unsigned* counters = nullptr;
    Tables tab[2];  // [PREC_F64], [PREC_F32]
    bool have_wfc = false;
    bool pending_scale = false;  // scal[kScale] must multiply psi
    std::map<GraphKey, Segment> graphs;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    long launches = 0;  // kernels enqueued in the current evolve call
    double last_energy = 0.0;  // energy of the latest check (GPUE's "energy" key)
};

namespace {

// device scalar slots
enum { kScale = 0, kEkin = 1, kEreal = 2, kNorm = 3, kNScal = 8 };
// counter slots (one per reduction that may be in flight in a graph)
enum { kCtrNorm = 0, kCtrEkin = 1, kCtrEreal = 2, kCtrMisc = 3, kNCtr = 8 };

gpue_status fail(gpue_ctx* c, gpue_status st, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return st;
}

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(c, e_ == cudaErrorMemoryAllocation ? GPUE_ERR_OUT_OF_MEMORY      \
                                                           : GPUE_ERR_CUDA,              \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,       \
                        __LINE__);                                                       \
    } while (0)

size_t elem_size(int prec) { return prec == GPUE_PREC_FP32 ? 8 : 16; }

// generate_p_space for one axis (src/operators.cu:336-343; init.cu:140-161)
void build_axis(Axis& a, int n, double xmax, bool active) {
    a.n = n;
    a.xmax = xmax;
    a.x.assign(n, 0.0);
    a.p.assign(n, 0.0);
    if (!active) {
        a.dx = 1.0;
        return;
    }
    a.dx = xmax / (n >> 1);
    const double dp = kPI / xmax;
    const double pmax = (kPI / xmax) * (n >> 1);
    for (int i = 0; i < n / 2; ++i) {
        a.x[i] = -xmax + i * a.dx;
        a.x[i + n / 2] = i * a.dx;
        a.p[i] = i * dp;
        a.p[i + n / 2] = -pmax + i * dp;
    }
}

bool gauge_active(const gpue_ctx* c) {
    return c->p.corotating && c->p.gauge == GPUE_GAUGE_ROTATION && c->p.omega != 0.0;
}

// A = (ax_coef * y, ay_coef * x, 0) for the rotation gauge (krotation_Ax/Ay,
// src/operators.cu:630-647); zero for the constant gauge.
void gauge_coefs(const gpue_ctx* c, double& axc, double& ayc) {
    if (c->p.gauge == GPUE_GAUGE_ROTATION) {
        axc = -c->p.omega * c->p.omegaX;
        ayc = c->p.omega * c->p.omegaY;
    } else {
        axc = ayc = 0.0;
    }
}

// Per-axis real V (kharmonic_V, src/operators.cu:994-1008, split by axis;
// the m|A|^2/2 term of the rotation gauge is separable too).
void axis_potential(const gpue_ctx* c, int a, std::vector<double>& v) {
    const gpue_params& p = c->p;
    const Axis& A = c->ax[a];
    double axc, ayc;
    gauge_coefs(c, axc, ayc);
    v.assign(A.n, 0.0);
    for (int i = 0; i < A.n; ++i) {
        const double x = A.x[i];
        double t = 0.0;
        if (a == 0) {
            const double vx = p.omegaX * (x + p.x0_shift);
            const double ay = ayc * x;  // Ay depends on x
            t = vx * vx + ay * ay;
        } else if (a == 1) {
            const double vy = p.gammaY * p.omegaY * (x + p.y0_shift);
            const double axv = axc * x;  // Ax depends on y
            t = vy * vy + axv * axv;
        } else if (c->dim == 3) {
            const double vz = p.omegaZ * (x + p.z0_shift);
            t = vz * vz;
        }
        v[i] = 0.5 * p.mass * t;
    }
}

template <typename T>
struct HostCx {
    T x, y;
};

// Build tables for precision `prec` and time type gstate (aux_fields,
// src/operators.cu:1069-1111, per axis).
gpue_status build_tables(gpue_ctx* c, int prec, int gstate) {
    Tables& tb = c->tab[prec];
    if (tb.built_for == gstate) return GPUE_OK;
    const gpue_params& p = c->p;
    const size_t es = elem_size(prec);
    // layout: per axis [vfac n][kfac n][tw n] complex, then [pos n][mom n][vreal n] double
    size_t off = 0;
    size_t offs[3][6];
    for (int a = 0; a < 3; ++a) {
        const int n = c->ax[a].n;
        for (int k = 0; k < 3; ++k) {
            offs[a][k] = off;
            off += ((n * es + 255) / 256) * 256;
        }
        for (int k = 3; k < 6; ++k) {
            offs[a][k] = off;
            off += ((n * 8 + 255) / 256) * 256;
        }
    }
    if (!tb.buf) CK(cudaMalloc(&tb.buf, off));
    std::vector<unsigned char> h(off, 0);
    for (int a = 0; a < 3; ++a) {
        const Axis& A = c->ax[a];
        const int n = A.n;
        std::vector<double> va;
        axis_potential(c, a, va);
        for (int i = 0; i < n; ++i) {
            const double K = (p.hbar * p.hbar / (2 * p.mass)) * (A.p[i] * A.p[i]);
            double vr, vi, kr, ki;
            if (gstate == 0) {
                vr = std::exp(-va[i] * (p.gdt / (2 * p.hbar)));
                vi = 0.0;
                kr = std::exp(-K * (p.gdt / p.hbar));
                ki = 0.0;
            } else {
                vr = std::cos(-va[i] * (p.dt / (2 * p.hbar)));
                vi = std::sin(-va[i] * (p.dt / (2 * p.hbar)));
                kr = std::cos(-K * (p.dt / p.hbar));
                ki = std::sin(-K * (p.dt / p.hbar));
            }
            const long double ang = -2.0L * 3.141592653589793238462643383279L * i / n;
            const double twr = (double)cosl(ang), twi = (double)sinl(ang);
            if (prec == GPUE_PREC_FP32) {
                ((HostCx<float>*)(h.data() + offs[a][0]))[i] = {(float)vr, (float)vi};
                ((HostCx<float>*)(h.data() + offs[a][1]))[i] = {(float)kr, (float)ki};
                ((HostCx<float>*)(h.data() + offs[a][2]))[i] = {(float)twr, (float)twi};
            } else {
                ((HostCx<double>*)(h.data() + offs[a][0]))[i] = {vr, vi};
                ((HostCx<double>*)(h.data() + offs[a][1]))[i] = {kr, ki};
                ((HostCx<double>*)(h.data() + offs[a][2]))[i] = {twr, twi};
            }
            ((double*)(h.data() + offs[a][3]))[i] = A.x[i];
            ((double*)(h.data() + offs[a][4]))[i] = A.p[i];
            ((double*)(h.data() + offs[a][5]))[i] = va[i];
        }
    }
    CK(cudaMemcpyAsync(tb.buf, h.data(), off, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    unsigned char* b = (unsigned char*)tb.buf;
    for (int a = 0; a < 3; ++a) {
        tb.vfac[a] = b + offs[a][0];
        tb.kfac[a] = b + offs[a][1];
        tb.tw[a] = b + offs[a][2];
        tb.pos[a] = (const double*)(b + offs[a][3]);
        tb.mom[a] = (const double*)(b + offs[a][4]);
        tb.vreal[a] = (const double*)(b + offs[a][5]);
    }
    tb.built_for = gstate;
    return GPUE_OK;
}

// ---------------------------------------------------------------- passes --

struct LPass {
    int axis;
    std::vector<int> ops;
    int red;          // RED_NONE / RED_NORM / RED_SUM
    int red_slot;     // scalar slot for the result
    int ctr;          // counter slot
    bool store = true;
    bool to_scratch = false;   // out = scratch
    bool from_scratch = false; // in = scratch
    double gauge_dt = 0;       // for OP_GAUGE
};

struct LaunchCfg {
    const PassKernel* k;
    int threads, blocks;
    size_t smem;
};

gpue_status pass_launch_cfg(gpue_ctx* c, int prec, int axis, LaunchCfg& lc) {
    const int n = c->ax[axis].n;
    const PassKernel* k = find_pass_kernel(prec, n);
    if (!k) return fail(c, GPUE_ERR_UNSUPPORTED, "no FFT plan for length %d", n);
    long nlines = c->N / n;
    int C;
    if (axis == 0) {
        C = 128 / k->p;
        if (C < 1) C = 1;
    } else {
        const int min_c = (32 + k->elem - 1) / k->elem;  // one 32-byte sector per row
        C = 128 / k->p;
        if (C < min_c) C = min_c;
        if (C * k->p > kMaxPassThreads) C = kMaxPassThreads / k->p;
        while (C > 1 && c->ax[0].n % C) C >>= 1;
    }
    while (C > 1 && nlines % C) C >>= 1;
    lc.k = k;
    lc.threads = C * k->p;
    lc.blocks = (int)(nlines / C);
    const size_t tsz = k->elem / 2;
    lc.smem = (size_t)C * 2 * k->ls * tsz;
    const size_t red_need = 2 * ((lc.threads + 31) / 32) * sizeof(double);
    if (lc.smem < red_need) lc.smem = red_need;
    return GPUE_OK;
}

gpue_status set_smem_attr(gpue_ctx* c, const LaunchCfg& lc, int axis) {
    void* fn = axis == 0 ? (void*)lc.k->row : (void*)lc.k->col;
    if (lc.smem > 48 * 1024)
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lc.smem));
    return GPUE_OK;
}

gpue_status launch_pass(gpue_ctx* c, int prec, const LPass& lp, int gstate) {
    LaunchCfg lc;
    gpue_status st = pass_launch_cfg(c, prec, lp.axis, lc);
    if (st) return st;
    if (lp.red != RED_NONE && lc.blocks > c->partials_cap)
        return fail(c, GPUE_ERR_INVALID_ARG, "reduction grid %d exceeds scratch", lc.blocks);
    const Tables& tb = c->tab[prec];
    const gpue_params& p = c->p;
    PassArgs a;
    std::memset(&a, 0, sizeof a);
    void* psi = (prec == c->prec) ? c->psi : nullptr;
    a.in = lp.from_scratch ? c->scratch : psi;
    a.out = lp.to_scratch ? c->scratch : (lp.from_scratch ? c->scratch : psi);
    a.axis = lp.axis;
    a.nx = c->ax[0].n;
    a.ny = c->ax[1].n;
    a.nz = c->ax[2].n;
    a.nops = (int)lp.ops.size();
    for (int i = 0; i < a.nops; ++i) a.ops[i] = lp.ops[i];
    a.store = lp.store ? 1 : 0;
    a.gstate = gstate;
    a.gpe = p.gpe;
    const double Dt = gstate == 0 ? p.gdt : p.dt;
    a.nl_coef = (p.interaction * p.gDenConst) * ((0.5 * Dt) / p.hbar);
    double axc, ayc;
    gauge_coefs(c, axc, ayc);
    if (lp.axis == 0) {
        a.gauge_coef = axc;
        a.gauge_src = 1;
    } else if (lp.axis == 1) {
        a.gauge_coef = ayc;
        a.gauge_src = 0;
    } else {
        a.gauge_coef = 0.0;
        a.gauge_src = 0;
    }
    a.gauge_dt = lp.gauge_dt;
    a.kin_coef = p.hbar * p.hbar / (2 * p.mass);
    for (int i = 0; i < 3; ++i) {
        a.vfac[i] = tb.vfac[i];
        a.kfac[i] = tb.kfac[i];
        a.pos[i] = tb.pos[i];
        a.mom[i] = tb.mom[i];
    }
    a.tw = tb.tw[lp.axis];
    a.inv_sqrt_n = 1.0 / std::pow((double)c->ax[lp.axis].n, 0.5);
    a.red.kind = lp.red;
    a.red.partials = c->partials;
    a.red.counter = c->counters + lp.ctr;
    a.red.out = c->scal + lp.red_slot;
    a.red.dV = c->dV;
    a.scale_in = c->scal + kScale;
    void (*fn)(PassArgs) = lp.axis == 0 ? lc.k->row : lc.k->col;
    fn<<<lc.blocks, lc.threads, lc.smem, c->stream>>>(a);
    c->launches++;
    CK(cudaGetLastError());
    return GPUE_OK;
}

// Logical passes of step i (see the file header).
void step_passes(gpue_ctx* c, int i, int gstate, bool scale_first, double rexp,
                 std::vector<LPass>& out) {
    const bool imag = gstate == 0;
    const bool g = gauge_active(c);
    const double gdt = imag ? c->p.gdt * rexp : c->p.dt;
    auto P = [&](int axis, std::vector<int> ops) {
        LPass lp;
        lp.axis = axis;
        lp.ops = ops;
        lp.red = RED_NONE;
        lp.red_slot = 0;
        lp.ctr = 0;
        lp.gauge_dt = gdt;
        return lp;
    };
    std::vector<LPass> s;
    std::vector<int> first;
    if (scale_first) first.push_back(OP_SCALE);
    first.push_back(OP_VHALF);
    first.push_back(OP_FFT_F);
    const bool flip = (i % 2) != 0;
    if (c->dim == 2) {
        s.push_back(P(0, first));
        s.push_back(P(1, {OP_FFT_F, OP_KPHASE, OP_FFT_I}));
        if (g && flip) {
            s.push_back(P(0, {OP_FFT_I, OP_VHALF, OP_FFT_F, OP_GAUGE, OP_FFT_I}));
            s.push_back(P(1, {OP_FFT_F, OP_GAUGE, OP_FFT_I}));
        } else if (g) {
            s.push_back(P(0, {OP_FFT_I, OP_VHALF}));
            s.push_back(P(1, {OP_FFT_F, OP_GAUGE, OP_FFT_I}));
            s.push_back(P(0, {OP_FFT_F, OP_GAUGE, OP_FFT_I}));
        } else {
            s.push_back(P(0, {OP_FFT_I, OP_VHALF}));
        }
    } else {
        s.push_back(P(0, first));
        s.push_back(P(1, {OP_FFT_F}));
        s.push_back(P(2, {OP_FFT_F, OP_KPHASE, OP_FFT_I}));
        s.push_back(P(1, {OP_FFT_I}));
        // Az = 0 for the rotation gauge: the z gauge pass is the identity
        if (g && flip) {
            s.push_back(P(0, {OP_FFT_I, OP_VHALF, OP_FFT_F, OP_GAUGE, OP_FFT_I}));
            s.push_back(P(1, {OP_FFT_F, OP_GAUGE, OP_FFT_I}));
        } else if (g) {
            s.push_back(P(0, {OP_FFT_I, OP_VHALF}));
            s.push_back(P(1, {OP_FFT_F, OP_GAUGE, OP_FFT_I}));
            s.push_back(P(0, {OP_FFT_F, OP_GAUGE, OP_FFT_I}));
        } else {
            s.push_back(P(0, {OP_FFT_I, OP_VHALF}));
        }
    }
    if (imag) {
        LPass& last = s.back();
        last.ops.push_back(OP_NORM);
        last.red = RED_NORM;
        last.red_slot = kScale;
        last.ctr = kCtrNorm;
    }
    for (auto& x : s) out.push_back(x);
}

// Fuse adjacent passes along the same axis when nothing global lies between.
void fuse(std::vector<LPass>& v) {
    std::vector<LPass> o;
    for (auto& p : v) {
        if (!o.empty()) {
            LPass& q = o.back();
            bool has_scale = false, q_gauge = false, p_gauge = false;
            for (int op : p.ops) has_scale |= (op == OP_SCALE), p_gauge |= (op == OP_GAUGE);
            for (int op : q.ops) q_gauge |= (op == OP_GAUGE);
            if (q.axis == p.axis && q.red == RED_NONE && !has_scale && q.store && p.store &&
                !q.to_scratch && !p.from_scratch && !(q_gauge && p_gauge) &&
                q.ops.size() + p.ops.size() <= (size_t)kMaxOps) {
                for (int op : p.ops) q.ops.push_back(op);
                q.red = p.red;
                q.red_slot = p.red_slot;
                q.ctr = p.ctr;
                if (p_gauge) q.gauge_dt = p.gauge_dt;
                continue;
            }
        }
        o.push_back(p);
    }
    v.swap(o);
}

// Energy passes: kinetic sum K|psi_k|^2 via a forward transform into scratch,
// and the real-space terms.  scale_pending applies the deferred renorm.
gpue_status launch_energy(gpue_ctx* c, int prec, int gstate, bool scale_pending) {
    std::vector<LPass> v;
    auto P = [&](int axis, std::vector<int> ops) {
        LPass lp;
        lp.axis = axis;
        lp.ops = ops;
        lp.red = RED_NONE;
        lp.red_slot = 0;
        lp.ctr = 0;
        return lp;
    };
    std::vector<int> f;
    if (scale_pending) f.push_back(OP_SCALE);
    f.push_back(OP_FFT_F);
    LPass x = P(0, f);
    x.to_scratch = true;
    v.push_back(x);
    if (c->dim == 3) {
        LPass y = P(1, {OP_FFT_F});
        y.from_scratch = true;
        v.push_back(y);
    }
    LPass last = P(c->dim == 3 ? 2 : 1, {OP_FFT_F, OP_EKIN});
    last.from_scratch = true;
    last.store = false;
    last.red = RED_SUM;
    last.red_slot = kEkin;
    last.ctr = kCtrEkin;
    v.push_back(last);
    for (auto& lp : v) {
        gpue_status st = launch_pass(c, prec, lp, gstate);
        if (st) return st;
    }
    const Tables& tb = c->tab[prec];
    EnergyArgs e;
    std::memset(&e, 0, sizeof e);
    e.psi = c->psi;
    e.N = c->N;
    e.nx = c->ax[0].n;
    e.ny = c->ax[1].n;
    e.nz = c->ax[2].n;
    e.dim = c->dim;
    e.scale = scale_pending ? c->scal + kScale : nullptr;
    for (int i = 0; i < 3; ++i) {
        e.vreal[i] = tb.vreal[i];
        e.pos[i] = tb.pos[i];
    }
    e.gN = c->p.interaction * c->p.gDenConst;
    e.gpe = c->p.gpe;
    double axc, ayc;
    gauge_coefs(c, axc, ayc);
    e.lterm = (c->p.corotating && c->dim > 1 && (axc != 0.0 || ayc != 0.0)) ? 1 : 0;
    e.ax_coef = axc;
    e.ay_coef = ayc;
    e.dx = c->ax[0].dx;
    e.dy = c->ax[1].dx;
    e.dz = c->ax[2].dx;
    e.hbar = c->p.hbar;
    e.red.kind = RED_SUM;
    e.red.partials = c->partials + (c->partials_cap - 2048);
    e.red.counter = c->counters + kCtrEreal;
    e.red.out = c->scal + kEreal;
    e.red.dV = c->dV;
    const int blocks = 148 * 4;
    if (prec == GPUE_PREC_FP32) k_energy_real<float><<<blocks, 256, 0, c->stream>>>(e);
    else k_energy_real<double><<<blocks, 256, 0, c->stream>>>(e);
    c->launches++;
    CK(cudaGetLastError());
    return GPUE_OK;
}

gpue_status read_energy(gpue_ctx* c, double* E) {
    double h[kNScal];
    CK(cudaMemcpyAsync(h, c->scal, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *E = (h[kEkin] + h[kEreal]) * c->dV;
    return GPUE_OK;
}

gpue_status apply_pending_scale(gpue_ctx* c) {
    if (!c->pending_scale) return GPUE_OK;
    if (c->prec == GPUE_PREC_FP32)
        k_scale<float><<<148 * 8, 256, 0, c->stream>>>(c->psi, c->N, c->scal + kScale);
    else
        k_scale<double><<<148 * 8, 256, 0, c->stream>>>(c->psi, c->N, c->scal + kScale);
    c->launches++;
    CK(cudaGetLastError());
    c->pending_scale = false;
    return GPUE_OK;
}

// Enqueue steps [i0, i1) (+ energy passes after the last one when asked).
gpue_status enqueue_steps(gpue_ctx* c, int i0, int i1, int gstate, bool scale_first,
                          const std::vector<double>& rexp, bool energy_after) {
    std::vector<LPass> v;
    for (int i = i0; i < i1; ++i)
        step_passes(c, i, gstate, scale_first && i == i0, rexp.empty() ? 1.0 : rexp[i], v);
    if (gstate != 0) fuse(v);
    for (auto& lp : v) {
        gpue_status st = launch_pass(c, c->prec, lp, gstate);
        if (st) return st;
    }
    if (energy_after) {
        gpue_status st = launch_energy(c, c->prec, gstate, gstate == 0);
        if (st) return st;
    }
    return GPUE_OK;
}

gpue_status run_segment(gpue_ctx* c, int i0, int i1, int gstate, bool scale_first,
                        const std::vector<double>& rexp, bool energy_after, bool use_graph) {
    if (!use_graph || !rexp.empty())
        return enqueue_steps(c, i0, i1, gstate, scale_first, rexp, energy_after);
    GraphKey key{gstate, i0 % 2, i1 - i0, scale_first ? 1 : 0, energy_after ? 1 : 0};
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
        long before = c->launches;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        gpue_status st = enqueue_steps(c, i0, i1, gstate, scale_first, rexp, energy_after);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        CK(ce);
        Segment seg;
        ce = cudaGraphInstantiate(&seg.exec, g, 0);
        cudaGraphDestroy(g);
        CK(ce);
        seg.launches = c->launches - before;
        c->launches = before;
        it = c->graphs.emplace(key, seg).first;
    }
    CK(cudaGraphLaunch(it->second.exec, c->stream));
    c->launches += it->second.launches;
    return GPUE_OK;
}

void destroy_graphs(gpue_ctx* c) {
    for (auto& kv : c->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->graphs.clear();
}

gpue_status norm_now(gpue_ctx* c, double* out) {
    RedArgs r;
    r.kind = RED_SUM;
    r.partials = c->partials + (c->partials_cap - 2048);
    r.counter = c->counters + kCtrMisc;
    r.out = c->scal + kNorm;
    r.dV = c->dV;
    if (c->prec == GPUE_PREC_FP32) k_norm<float><<<148 * 4, 256, 0, c->stream>>>(c->psi, c->N, r);
    else k_norm<double><<<148 * 4, 256, 0, c->stream>>>(c->psi, c->N, r);
    CK(cudaGetLastError());
    double h;
    CK(cudaMemcpyAsync(&h, c->scal + kNorm, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *out = h * c->dV;
    return GPUE_OK;
}

}  // namespace

// ================================================================= C ABI ==

extern "C" {

int gpue_abi_version(void) { return GPUE_B200_ABI_VERSION; }

int gpue_supported_length(int32_t precision, int32_t n) {
    return find_pass_kernel(precision == GPUE_PREC_FP32 ? PREC_F32 : PREC_F64, n) ? 1 : 0;
}

gpue_status gpue_default_params(gpue_params* p) {
    if (!p) return GPUE_ERR_INVALID_ARG;
    std::memset(p, 0, sizeof *p);
    // parseArgs defaults (src/parser.cu:14-67) and init()'s derived values
    // (src/init.cu:98-170) for the default 2D run with one atom
    const double HBAR = 1.05457148e-34, mass = 1.4431607e-25, a_s = 4.76e-9;
    p->dimnum = 2;
    p->xDim = p->yDim = 256;
    p->zDim = 1;
    p->hbar = HBAR;
    p->mass = mass;
    p->omegaX = p->omegaY = p->omegaZ = 6.283;
    p->gammaY = 1.0;
    p->interaction = 1.0;
    const double N = 1.0;
    p->gDenConst = N * 4 * HBAR * HBAR * kPI * (a_s / mass) *
                   std::sqrt(mass * p->omegaZ / (2 * kPI * HBAR));
    const double Rxy = std::pow(15.0, 0.2) * std::pow(N * a_s * std::sqrt(mass * p->omegaZ / HBAR), 0.2);
    const double a0x = std::sqrt(HBAR / (2 * mass * p->omegaX));
    const double a0y = std::sqrt(HBAR / (2 * mass * p->omegaY));
    p->xMax = 6 * Rxy * a0x;
    p->yMax = 6 * Rxy * a0y;
    p->zMax = 6 * Rxy * std::sqrt(HBAR / (2 * mass * p->omegaZ));
    p->gdt = p->dt = 1e-4;
    p->gauge = GPUE_GAUGE_ROTATION;
    p->ramp_type = 1;
    p->precision = GPUE_PREC_FP64;
    return GPUE_OK;
}

gpue_status gpue_ctx_create(const gpue_params* p, gpue_ctx** out) {
    if (!p || !out) return GPUE_ERR_INVALID_ARG;
    *out = nullptr;
    std::unique_ptr<gpue_ctx> cp(new gpue_ctx);
    gpue_ctx* c = cp.get();
    c->p = *p;
    c->dim = p->dimnum;
    c->prec = p->precision == GPUE_PREC_FP32 ? GPUE_PREC_FP32 : GPUE_PREC_FP64;
    if (c->dim != 2 && c->dim != 3)
        return GPUE_ERR_INVALID_ARG;
    const int nx = p->xDim, ny = p->yDim, nz = c->dim == 3 ? p->zDim : 1;
    if (nx < 2 || ny != nx || (c->dim == 3 && nz != nx)) return GPUE_ERR_INVALID_ARG;
    if (!(p->xMax > 0) || !(p->hbar > 0) || !(p->mass > 0)) return GPUE_ERR_INVALID_ARG;
    if (!gpue_supported_length(c->prec, nx)) return GPUE_ERR_UNSUPPORTED;
    build_axis(c->ax[0], nx, p->xMax, true);
    build_axis(c->ax[1], ny, p->dimnum > 1 ? p->yMax : 1.0, true);
    build_axis(c->ax[2], nz, p->zMax, c->dim == 3);
    c->N = (long)nx * ny * nz;
    c->dV = c->ax[0].dx * c->ax[1].dx * (c->dim == 3 ? c->ax[2].dx : 1.0);
    c->device = p->device;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    CK(cudaMalloc(&c->psi, c->N * elem_size(c->prec)));
    CK(cudaMalloc(&c->scratch, c->N * 16));
    CK(cudaMalloc(&c->scal, kNScal * sizeof(double)));
    c->partials_cap = c->N / nx + 4096;
    CK(cudaMalloc(&c->partials, c->partials_cap * sizeof(double2)));
    CK(cudaMalloc(&c->counters, kNCtr * sizeof(unsigned)));
    CK(cudaMemsetAsync(c->counters, 0, kNCtr * sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->scal, 0, kNScal * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->psi, 0, c->N * elem_size(c->prec), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    gpue_status st = build_tables(c, c->prec, 0);
    if (st) return st;
    for (int a = 0; a < c->dim; ++a) {
        LaunchCfg lc;
        st = pass_launch_cfg(c, c->prec, a, lc);
        if (st) return st;
        st = set_smem_attr(c, lc, a);
        if (st) return st;
    }
    *out = cp.release();
    return GPUE_OK;
}

gpue_status gpue_ctx_destroy(gpue_ctx* c) {
    if (!c) return GPUE_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    destroy_graphs(c);
    for (auto& t : c->tab)
        if (t.buf) cudaFree(t.buf);
    cudaFree(c->psi);
    cudaFree(c->scratch);
    cudaFree(c->scal);
    cudaFree(c->partials);
    cudaFree(c->counters);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return GPUE_OK;
}

const char* gpue_last_error(const gpue_ctx* c) { return c ? c->err.c_str() : ""; }

gpue_status gpue_set_operators(gpue_ctx* c, int32_t ev_type) {
    if (!c || (ev_type != 0 && ev_type != 1)) return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    return build_tables(c, c->prec, ev_type);
}

gpue_status gpue_set_wfc(gpue_ctx* c, const void* psi, int32_t mem, int32_t dtype) {
    if (!c || !psi || (mem != GPUE_MEM_HOST && mem != GPUE_MEM_DEVICE) ||
        (dtype != GPUE_C128 && dtype != GPUE_C64))
        return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    const int want = c->prec == GPUE_PREC_FP32 ? GPUE_C64 : GPUE_C128;
    const size_t in_bytes = c->N * (dtype == GPUE_C128 ? 16 : 8);
    const cudaMemcpyKind kind = mem == GPUE_MEM_HOST ? cudaMemcpyHostToDevice
                                                     : cudaMemcpyDeviceToDevice;
    if (dtype == want) {
        CK(cudaMemcpyAsync(c->psi, psi, in_bytes, kind, c->stream));
    } else {
        CK(cudaMemcpyAsync(c->scratch, psi, in_bytes, kind, c->stream));
        if (dtype == GPUE_C128)
            k_convert<double, float><<<148 * 8, 256, 0, c->stream>>>(c->scratch, c->psi, c->N);
        else
            k_convert<float, double><<<148 * 8, 256, 0, c->stream>>>(c->scratch, c->psi, c->N);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(c->stream));
    c->have_wfc = true;
    c->pending_scale = false;
    return GPUE_OK;
}

gpue_status gpue_get_wfc(gpue_ctx* c, void* psi, int32_t mem, int32_t dtype) {
    if (!c || !psi || (mem != GPUE_MEM_HOST && mem != GPUE_MEM_DEVICE) ||
        (dtype != GPUE_C128 && dtype != GPUE_C64))
        return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    gpue_status st = apply_pending_scale(c);
    if (st) return st;
    const int have = c->prec == GPUE_PREC_FP32 ? GPUE_C64 : GPUE_C128;
    const size_t out_bytes = c->N * (dtype == GPUE_C128 ? 16 : 8);
    const cudaMemcpyKind kind = mem == GPUE_MEM_HOST ? cudaMemcpyDeviceToHost
                                                     : cudaMemcpyDeviceToDevice;
    if (dtype == have) {
        CK(cudaMemcpyAsync(psi, c->psi, out_bytes, kind, c->stream));
    } else {
        if (have == GPUE_C64)
            k_convert<float, double><<<148 * 8, 256, 0, c->stream>>>(c->psi, c->scratch, c->N);
        else
            k_convert<double, float><<<148 * 8, 256, 0, c->stream>>>(c->psi, c->scratch, c->N);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(psi, c->scratch, out_bytes, kind, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return GPUE_OK;
}

gpue_status gpue_energy(gpue_ctx* c, double* E) {
    if (!c || !E) return GPUE_ERR_INVALID_ARG;
    if (!c->have_wfc) return fail(c, GPUE_ERR_STATE, "no wavefunction set");
    CK(cudaSetDevice(c->device));
    const int gs = c->tab[c->prec].built_for < 0 ? 0 : c->tab[c->prec].built_for;
    gpue_status st = launch_energy(c, c->prec, gs, c->pending_scale);
    if (st) return st;
    return read_energy(c, E);
}

gpue_status gpue_norm(gpue_ctx* c, double* out) {
    if (!c || !out) return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    gpue_status st = apply_pending_scale(c);
    if (st) return st;
    return norm_now(c, out);
}

gpue_status gpue_ctx_stream(gpue_ctx* c, void** s) {
    if (!c || !s) return GPUE_ERR_INVALID_ARG;
    *s = (void*)c->stream;
    return GPUE_OK;
}

gpue_status gpue_ctx_wfc_device(gpue_ctx* c, void** psi, int32_t* dtype) {
    if (!c || !psi || !dtype) return GPUE_ERR_INVALID_ARG;
    *psi = c->psi;
    *dtype = c->prec == GPUE_PREC_FP32 ? GPUE_C64 : GPUE_C128;
    return GPUE_OK;
}

gpue_status gpue_evolve(gpue_ctx* c, int32_t nsteps, int32_t gstate,
                        const gpue_evolve_opts* opts, gpue_evolve_result* res) {
    if (!c || nsteps < 0 || (gstate != 0 && gstate != 1)) return GPUE_ERR_INVALID_ARG;
    if (!c->have_wfc) return fail(c, GPUE_ERR_STATE, "no wavefunction set");
    CK(cudaSetDevice(c->device));
    gpue_evolve_opts o;
    std::memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    if (o.polish_steps > 0 && c->prec == GPUE_PREC_FP64) o.polish_steps = 0;
    if (o.no_sync && o.energy_calc_steps > 0)
        return fail(c, GPUE_ERR_INVALID_ARG, "no_sync excludes energy checks");
    gpue_status st = build_tables(c, c->prec, gstate);
    if (st) return st;
    c->launches = 0;
    // ramp exponent per step (src/evolution.cu:409-427): GPUE raises the gauge
    // tables to omega_0 every step, so the exponent at step i is cumulative
    // absolute step indices [off, last): time = Dt*i and the gauge order i%2
    const int off = o.step_offset > 0 ? o.step_offset : 0;
    const int last = off + nsteps;
    std::vector<double> rexp;
    if (c->p.ramp && gstate == 0 && gauge_active(c)) {
        rexp.resize(last);
        double r = 1.0;
        for (int i = 0; i < last; ++i) {
            double w0;
            if (c->p.ramp_type == 1) w0 = (i == 0) ? c->p.omega : (double)i / (double)(i + 1);
            else w0 = (i == 0) ? c->p.omega / (double)last : (double)(i + 1) / (double)i;
            r *= w0;
            rexp[i] = r;
        }
    }
    const int every = o.energy_calc_steps;
    const int chunk = o.graph_chunk > 0 ? o.graph_chunk : 64;
    CK(cudaEventRecord(c->ev0, c->stream));
    // GPUE compares with the energy stored by the previous check
    // (par.dval("energy")), which a sliced run carries across calls
    double old_energy = off > 0 ? c->last_energy : 0.0, energy = NAN;
    int n_en = 0, done = 0, early = 0;
    int i = off;
    // the first imaginary step has no deferred scale to apply
    bool scale_next = (gstate == 0) && c->pending_scale;
    while (i < last) {
        // segments of at most `chunk` steps, ending right after each energy
        // check step (i % every == 0, as GPUE's evolve checks)
        int seg_end = i + chunk < last ? i + chunk : last;
        bool check = false;
        if (every > 0) {
            const int nc = ((i + every - 1) / every) * every;
            if (nc < last && nc + 1 <= seg_end) {
                seg_end = nc + 1;
                check = true;
            }
        }
        st = run_segment(c, i, seg_end, gstate, scale_next, rexp, check, true);
        if (st) return st;
        if (gstate == 0) {
            scale_next = true;
            c->pending_scale = true;
        }
        i = seg_end;
        done = i - off;
        if (check) {
            st = read_energy(c, &energy);
            if (st) return st;
            n_en++;
            c->last_energy = energy;
            const int step = i - 1;
            bool stop = o.threshold_abs
                            ? std::fabs(old_energy - energy) < o.energy_calc_threshold
                            : std::fabs(old_energy - energy) < o.energy_calc_threshold * old_energy;
            if (step != 0 && stop && gstate == 0) {
                early = 1;
                break;
            }
            old_energy = energy;
        }
    }
    st = apply_pending_scale(c);
    if (st) return st;
    if (o.no_sync) {
        if (res) {
            std::memset(res, 0, sizeof *res);
            res->steps_done = done;
            res->energy = NAN;
            res->kernel_launches = c->launches;
        }
        return GPUE_OK;
    }
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (res) {
        std::memset(res, 0, sizeof *res);
        res->steps_done = done;
        res->early_stop = early;
        res->n_energies = n_en;
        res->energy = energy;
        res->device_ms = ms;
        res->kernel_launches = c->launches;
        double nrm = 0;
        st = norm_now(c, &nrm);
        if (st) return st;
        res->norm = nrm;
    }
    return GPUE_OK;
}

}  // extern "C"

namespace gpue {

const PassKernel* find_pass_kernel(int prec, int n) {
    int cnt = 0;
    const PassKernel* t = prec == PREC_F32 ? pass_table_f32(&cnt) : pass_table_f64(&cnt);
    for (int i = 0; i < cnt; ++i)
        if (t[i].n == n) return &t[i];
    return nullptr;
}

}  // namespace gpue
