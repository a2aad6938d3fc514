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
// fused when they share an axis (no renormalisation lies between them).  The
// z gauge pass is left out: Az = 0 for the rotation gauge.
//
// An FP32-form context keeps an FP64 shadow of the state for the polishing
// steps that end an imaginary-time run; after a polish the FP64 state is the
// authoritative one until the next FP32 evolve.


#include <cstdlib>

#include "engine_internal.h"

using namespace gpue;
using namespace gpue_eng;

namespace gpue_eng {

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

size_t elem_size(int prec) { return prec == GPUE_PREC_FP32 ? 8 : 16; }
int kprec(int prec) { return prec == GPUE_PREC_FP32 ? PREC_F32 : PREC_F64; }

void* state_of(gpue_ctx* c, int prec) {
    return prec == c->prec ? c->psi : c->psi64;
}

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

// Does the gauge pass along `axis` change the state?  Preset rotation: x and
// y when omega != 0; parameter-file fields: a time-dependent expression, or a
// static table that is not identically zero.
bool axis_gauge_active(const gpue_ctx* c, int axis) {
    if (c->prog_off[2 + axis] >= 0) return true;
    if (c->use_atab) return c->atab_nonzero[axis];
    return axis < 2 && gauge_active(c);
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

// Build tables for precision `prec` and time type gstate (aux_fields,
// src/operators.cu:1069-1111, per axis).  Factors are FP64 in both forms;
// the DFT twiddles are in the storage precision.
gpue_status build_tables(gpue_ctx* c, int prec, int gstate) {
    Tables& tb = c->tab[prec];
    if (tb.built_for == gstate) return GPUE_OK;
    const gpue_params& p = c->p;
    auto al = [](size_t b) { return ((b + 255) / 256) * 256; };
    // per axis: [vfac][kfac] double2, [tw] FP64 complex or FP32 (hi, lo) pairs,
    // [pos][mom][vreal] double, [vd][kd] float2
    size_t off = 0;
    size_t offs[3][8];
    for (int a = 0; a < 3; ++a) {
        const size_t n = c->ax[a].n;
        offs[a][0] = off; off += al(n * 16);
        offs[a][1] = off; off += al(n * 16);
        offs[a][2] = off; off += al(n * 16);  // FP64 twiddles, or FP32 (hi, lo) pairs
        for (int k = 3; k < 6; ++k) { offs[a][k] = off; off += al(n * 8); }
        for (int k = 6; k < 8; ++k) { offs[a][k] = off; off += al(n * 8); }
    }
    if (!tb.buf) CK(cudaMalloc(&tb.buf, off));
    std::vector<unsigned char> h(off, 0);
    // factor - 1 of exp(-a) (imaginary time) or exp(-i a) (real time), formed
    // without cancellation in long double and rounded once to FP32
    auto fdelta = [&](long double ang, float* d) {
        if (gstate == 0) {
            d[0] = (float)expm1l(-ang);
            d[1] = 0.f;
        } else {
            const long double h = sinl(0.5L * ang);
            d[0] = (float)(-2.0L * h * h);
            d[1] = (float)(-sinl(ang));
        }
    };
    for (int a = 0; a < 3; ++a) {
        const Axis& A = c->ax[a];
        const int n = A.n;
        std::vector<double> va;
        axis_potential(c, a, va);
        double* vf = (double*)(h.data() + offs[a][0]);
        double* kf = (double*)(h.data() + offs[a][1]);
        float* vd = (float*)(h.data() + offs[a][6]);
        float* kd = (float*)(h.data() + offs[a][7]);
        for (int i = 0; i < n; ++i) {
            const double K = (p.hbar * p.hbar / (2 * p.mass)) * (A.p[i] * A.p[i]);
            const double Dt = gstate == 0 ? p.gdt : p.dt;
            fdelta((long double)va[i] * ((long double)Dt / (2.0L * p.hbar)), vd + 2 * i);
            fdelta((long double)K * ((long double)Dt / p.hbar), kd + 2 * i);
            if (gstate == 0) {
                vf[2 * i] = std::exp(-va[i] * (p.gdt / (2 * p.hbar)));
                vf[2 * i + 1] = 0.0;
                kf[2 * i] = std::exp(-K * (p.gdt / p.hbar));
                kf[2 * i + 1] = 0.0;
            } else {
                vf[2 * i] = std::cos(-va[i] * (p.dt / (2 * p.hbar)));
                vf[2 * i + 1] = std::sin(-va[i] * (p.dt / (2 * p.hbar)));
                kf[2 * i] = std::cos(-K * (p.dt / p.hbar));
                kf[2 * i + 1] = std::sin(-K * (p.dt / p.hbar));
            }
            const long double ang = -2.0L * 3.141592653589793238462643383279L * i / n;
            const double twr = (double)cosl(ang), twi = (double)sinl(ang);
            if (prec == GPUE_PREC_FP32) {
                // one 16-byte entry per k: the rounded twiddle and its remainder
                float* tw = (float*)(h.data() + offs[a][2]);
                const float hr = (float)twr, hi = (float)twi;
                tw[4 * i] = hr;
                tw[4 * i + 1] = hi;
                tw[4 * i + 2] = (float)(twr - (double)hr);
                tw[4 * i + 3] = (float)(twi - (double)hi);
            } else {
                double* tw = (double*)(h.data() + offs[a][2]);
                tw[2 * i] = twr;
                tw[2 * i + 1] = twi;
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
        tb.vfac[a] = (const double2*)(b + offs[a][0]);
        tb.kfac[a] = (const double2*)(b + offs[a][1]);
        tb.tw[a] = b + offs[a][2];
        tb.pos[a] = (const double*)(b + offs[a][3]);
        tb.mom[a] = (const double*)(b + offs[a][4]);
        tb.vreal[a] = (const double*)(b + offs[a][5]);
        tb.vd[a] = (const float2*)(b + offs[a][6]);
        tb.kd[a] = (const float2*)(b + offs[a][7]);
    }
    tb.built_for = gstate;
    return GPUE_OK;
}

// ---------------------------------------------------------------- passes --

// Launch shape of plan k with C lines per tile and a persistent grid of
// (resident CTAs per SM) x SMs walking the tiles; false when C does not fit.
bool build_cfg(gpue_ctx* c, int prec, int axis, const PassKernel* k, int C, LaunchCfg& lc) {
    const long nlines = c->N / c->ax[axis].n;
    if (C < 1 || C * k->p > k->max_threads || nlines % C) return false;
    if (axis > 0 && c->ax[0].n % C) return false;  // a tile's lines are adjacent in x
    size_t smem = (size_t)C * k->ls * k->elem;
    const size_t red_need = 2 * ((C * k->p + 31) / 32) * sizeof(double);
    if (smem < red_need) smem = red_need;
    int max_smem = 48 * 1024;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (smem > (size_t)max_smem) return false;
    void* fns[6] = {(void*)k->row,       (void*)k->col,     (void*)k->row_batch,
                    (void*)k->col_batch, (void*)k->row_ext, (void*)k->col_ext};
    if (smem > 48 * 1024)
        for (void* f : fns)
            if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                cudaSuccess)
                return false;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, axis == 0 ? fns[0] : fns[1],
                                                      C * k->p, smem) != cudaSuccess)
        return false;
    if (per_sm < 1) return false;
    lc = LaunchCfg();
    lc.k = k;
    lc.lines = C;
    lc.threads = C * k->p;
    lc.ntiles = nlines / C;
    lc.smem = smem;
    long blocks = (long)per_sm * c->sms;
    if (blocks > lc.ntiles) blocks = lc.ntiles;
    lc.blocks = (int)blocks;
    return true;
}

// Lines per tile without tuning: 128 threads per tile for rows; for strided
// passes at least one 32-byte sector per row.
int default_lines(const gpue_ctx* c, int axis, const PassKernel* k) {
    const long nlines = c->N / c->ax[axis].n;
    int C;
    if (axis == 0) {
        C = 128 / k->p;
        if (C < 1) C = 1;
    } else {
        const int min_c = (32 + k->elem - 1) / k->elem;
        C = 128 / k->p;
        if (C < min_c) C = min_c;
        if (C * k->p > k->max_threads) C = k->max_threads / k->p;
        while (C > 1 && c->ax[0].n % C) C >>= 1;
    }
    while (C > 1 && nlines % C) C >>= 1;
    return C;
}

struct TuneKey {
    int prec, dim, n, axis;
    bool operator<(const TuneKey& o) const { return std::memcmp(this, &o, sizeof o) < 0; }
};
struct TuneChoice {
    int ra, rb, rc, p, lines;
    float us, default_us;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune;  // per process, guarded by g_tune_mu

bool cached_choice(const gpue_ctx* c, int prec, int axis, TuneChoice& out) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(TuneKey{prec, c->dim, c->ax[axis].n, axis});
    if (it == g_tune.end()) return false;
    out = it->second;
    return true;
}

gpue_status plan_axis(gpue_ctx* c, int prec, int axis) {
    LaunchCfg& lc = c->lc[prec][axis];
    const int n = c->ax[axis].n;
    const PassKernel* ks[8];
    const int nk = find_pass_kernels(kprec(prec), n, ks, 8);
    if (!nk) return fail(c, GPUE_ERR_UNSUPPORTED, "no FFT plan for length %d", n);
    TuneChoice tc;
    if (cached_choice(c, prec, axis, tc)) {
        for (int i = 0; i < nk; ++i)
            if (ks[i]->ra == tc.ra && ks[i]->rb == tc.rb && ks[i]->rc == tc.rc &&
                ks[i]->p == tc.p && build_cfg(c, prec, axis, ks[i], tc.lines, lc)) {
                lc.tuned = true;
                lc.us = tc.us;
                lc.default_us = tc.default_us;
                return GPUE_OK;
            }
    }
    if (!build_cfg(c, prec, axis, ks[0], default_lines(c, axis, ks[0]), lc))
        return fail(c, GPUE_ERR_CUDA, "no launch shape for length %d", n);
    return GPUE_OK;
}

gpue_status plan_plane(gpue_ctx* c, int prec) {
    PlaneCfg& pc = c->plane[prec];
    pc = PlaneCfg();
    const char* env = std::getenv("GPUE_PLANE");
    if (env && env[0] == '0') return GPUE_OK;
    if (c->dim != 3 || c->ax[0].n != c->ax[1].n) return GPUE_OK;
    const PlaneKernel* k = find_plane_kernel(kprec(prec), c->ax[0].n);
    if (!k) return GPUE_OK;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (k->smem > max_smem) return GPUE_OK;
    int ncl = 1 << 30;
    for (void (*fn)(PassArgs) : {k->fwd, k->inv}) {
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k->smem));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(k->cs);
        cfg.blockDim = dim3(k->threads);
        cfg.dynamicSmemBytes = k->smem;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = k->cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        CK(cudaOccupancyMaxActiveClusters(&n, fn, &cfg));
        ncl = std::min(ncl, n);
    }
    if (ncl < 1) return GPUE_OK;
    ncl = std::min(ncl, c->ax[2].n);
    pc.k = k;
    pc.blocks = ncl * k->cs;
    return GPUE_OK;
}

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links only the runtime)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// Allocates (once) and clears the work counters of a tile-stream pass.
gpue_status alloc_counters(gpue_ctx* c, TSCounters& t) {
    if (t.mem) return GPUE_OK;
    t.bytes = 16 + (size_t)c->ax[2].n * sizeof(int);
    CK(cudaMalloc(&t.mem, t.bytes));
    CK(cudaMemsetAsync(t.mem, 0, t.bytes, c->stream));
    return GPUE_OK;
}

EncodeTiled encode_tiled() {
    static EncodeTiled fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiled) nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

}  // namespace

gpue_status plan_zpass(gpue_ctx* c, int prec) {
    ZCfg& zc = c->zpass[prec];
    zc.k = nullptr;
    const char* env = std::getenv("GPUE_ZTMA");
    if (env && env[0] == '0') return GPUE_OK;
    if (c->dim != 3 || c->ax[0].n % 16 || c->ax[2].n > 256) return GPUE_OK;
    const ZPassKernel* k = find_zpass_kernel(kprec(prec), c->ax[2].n);
    EncodeTiled enc = encode_tiled();
    if (!k || !enc) return GPUE_OK;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (k->smem > max_smem) return GPUE_OK;
    CK(cudaFuncSetAttribute(k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k->smem));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k->fn, k->threads, k->smem));
    if (per_sm < 1) return GPUE_OK;
    // the field as nx x ny x nz elements of 8 bytes (one complex64 each); a
    // box is 16 x-columns of one y-row over all planes, landed with the
    // 128-byte swizzle (its rows are 16 x 8 = 128 bytes)
    const cuuint64_t dims[3] = {(cuuint64_t)c->ax[0].n, (cuuint64_t)c->ax[1].n,
                                (cuuint64_t)c->ax[2].n};
    const cuuint64_t strides[2] = {(cuuint64_t)c->ax[0].n * 8,
                                   (cuuint64_t)c->ax[0].n * c->ax[1].n * 8};
    const cuuint32_t box[3] = {16, 1, (cuuint32_t)c->ax[2].n};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (enc(&zc.tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, state_of(c, prec), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return GPUE_OK;
    gpue_status st = alloc_counters(c, zc.ctr);
    if (st) return st;
    const long tiles = (long)(c->ax[0].n / 16) * c->ax[1].n;
    zc.blocks = (int)std::min<long>((long)per_sm * c->sms, tiles);
    zc.k = k;
    return GPUE_OK;
}

gpue_status plan_xy(gpue_ctx* c, int prec) {
    XYCfg& xc = c->xy[prec];
    xc.k = nullptr;
    const char* env = std::getenv("GPUE_XY");
    if (env && env[0] == '0') return GPUE_OK;
    if (c->dim != 3 || c->ax[0].n != c->ax[1].n || c->ax[0].n > 256) return GPUE_OK;
    const XYKernel* k = find_xy_kernel(kprec(prec), c->ax[0].n);
    EncodeTiled enc = encode_tiled();
    if (!k || !enc) return GPUE_OK;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (k->smem > max_smem) return GPUE_OK;
    int per_sm = 1 << 30;
    for (const void* fn : {k->fwd, k->inv}) {
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k->smem));
        int n = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, k->threads, k->smem));
        per_sm = std::min(per_sm, n);
    }
    if (per_sm < 1) return GPUE_OK;
    const int n = c->ax[0].n;
    const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)c->ax[2].n};
    const cuuint64_t strides[2] = {(cuuint64_t)n * 8, (cuuint64_t)n * n * 8};
    // x-tiles: 16 whole rows, as they lie; y-tiles: 16 x-columns over all
    // y, landed with the 128-byte swizzle (rows of 16 x 8 = 128 bytes)
    const cuuint32_t boxx[3] = {(cuuint32_t)n, 16, 1}, boxy[3] = {16, (cuuint32_t)n, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    for (int w = 0; w < 2; ++w)
        if (enc(w ? &xc.tmy : &xc.tmx, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, state_of(c, prec),
                dims, strides, w ? boxy : boxx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                w ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_NONE,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return GPUE_OK;
    gpue_status st = alloc_counters(c, xc.ctr);
    if (st) return st;
    if (const char* lag = std::getenv("GPUE_XY_LAG")) xc.ctr.lag = std::max(1, std::atoi(lag));
    if (const char* w = std::getenv("GPUE_TEST_PLANE_WAIT")) xc.ctr.wait_extra = std::max(0, std::atoi(w));
    const long tiles = 2L * (n / 16) * c->ax[2].n;
    xc.blocks = (int)std::min<long>((long)per_sm * c->sms, tiles);
    xc.k = k;
    return GPUE_OK;
}

bool plane_ok(const gpue_ctx* c, int prec) {
    if (c->xy[prec].k && !c->ext)
        return !(c->p.corotating && (axis_gauge_active(c, 0) || axis_gauge_active(c, 1)));
    if (!c->plane[prec].k || c->ext) return false;
    return !(c->p.corotating && (axis_gauge_active(c, 0) || axis_gauge_active(c, 1)));
}

gpue_status make_pass_args(gpue_ctx* c, int prec, const LPass& lp, int gstate, PassArgs& a) {
    const bool plane = lp.axis >= kPlaneFwd;
    const int ax_i = plane ? 0 : lp.axis;  // the plane passes transform x (and y = x)
    const LaunchCfg& lc = c->lc[prec][ax_i];
    if (plane) {
        if (!c->plane[prec].k && !c->xy[prec].k)
        return fail(c, GPUE_ERR_STATE, "plane passes not planned");
    } else {
        if (!lc.k) return fail(c, GPUE_ERR_STATE, "axis %d not planned", lp.axis);
        if (lp.red != RED_NONE && lc.ntiles > c->partials_cap - kAuxPartials &&
            lc.blocks > c->partials_cap - kAuxPartials)
            return fail(c, GPUE_ERR_INVALID_ARG, "reduction grid %d exceeds scratch", lc.blocks);
    }
    const Tables& tb = c->tab[prec];
    const gpue_params& p = c->p;
    std::memset(&a, 0, sizeof a);
    void* psi = state_of(c, prec);
    a.in = lp.from_scratch ? c->scratch : psi;
    a.out = (lp.to_scratch || lp.from_scratch) ? c->scratch : psi;
    a.axis = lp.axis;
    a.nx = c->ax[0].n;
    a.ny = c->ax[1].n;
    a.nz = c->ax[2].n;
    a.ntiles = plane ? c->ax[2].n : lc.ntiles;
    a.nops = (int)lp.ops.size();
    for (int i = 0; i < a.nops; ++i) a.ops[i] = lp.ops[i];
    a.store = lp.store ? 1 : 0;
    a.gstate = gstate;
    a.gpe = p.gpe;
    const double Dt = gstate == 0 ? p.gdt : p.dt;
    a.nl_coef = (p.interaction * p.gDenConst) * ((0.5 * Dt) / p.hbar);
    a.kscale = 1.0 / (double)c->N;
    a.gscale = 1.0 / (double)c->ax[ax_i].n;
    double axc, ayc;
    gauge_coefs(c, axc, ayc);
    a.gauge_coef = lp.axis == 0 ? axc : lp.axis == 1 ? ayc : 0.0;
    a.gauge_src = lp.axis == 0 ? 1 : 0;
    a.gauge_dt = lp.gauge_dt;
    a.dmom = c->ax[ax_i].n > 1 ? c->ax[ax_i].p[1] : 0.0;
    a.kin_coef = p.hbar * p.hbar / (2 * p.mass);
    for (int i = 0; i < 3; ++i) {
        a.vfac[i] = tb.vfac[i];
        a.kfac[i] = tb.kfac[i];
        a.vd[i] = tb.vd[i];
        a.kd[i] = tb.kd[i];
        a.pos[i] = tb.pos[i];
        a.mom[i] = tb.mom[i];
    }
    a.tw = tb.tw[ax_i];
    a.red.kind = lp.red;
    a.red.partials = c->partials;
    a.red.counter = c->counters + lp.ctr;
    a.red.out = c->scal + lp.red_slot;
    a.red.target = c->scal + lp.red_target;
    a.scale_in = c->scal + lp.scale_slot;
    a.kscale_in = lp.kscale_slot >= 0 ? c->scal + lp.kscale_slot : nullptr;
    a.hbar = p.hbar;
    a.step_dt = Dt;
    a.time = lp.time;
    // evolve() passes dx, and dy/dz only where the axis exists (1 otherwise)
    a.grid_d[0] = c->ax[0].dx;
    a.grid_d[1] = c->dim > 1 ? c->ax[1].dx : 1.0;
    a.grid_d[2] = c->dim > 2 ? c->ax[2].dx : 1.0;
    if (c->ext) {
        a.vtab = c->vtab;
        for (int i = 0; i < 3; ++i) a.atab[i] = c->use_atab ? c->atab[i] : nullptr;
        auto prog = [&](int k, const AstInstr*& pp, int& n) {
            pp = c->prog_off[k] >= 0 ? c->progs + c->prog_off[k] : nullptr;
            n = c->prog_len[k];
        };
        prog(0, a.prog_v, a.nprog_v);
        prog(1, a.prog_k, a.nprog_k);
        for (int i = 0; i < 3; ++i) prog(2 + i, a.prog_a[i], a.nprog_a[i]);
    }
    a.active = c->dflags;
    a.err = c->dflags + 3;
    return GPUE_OK;
}

// pdl: the previous operation in the stream is a pass kernel
bool tile_pass(gpue_ctx* c, int prec, const LPass& lp, const PassArgs& a, TileLaunch& t) {
    if (lp.axis >= kPlaneFwd && c->xy[prec].k) {
        const XYCfg& xc = c->xy[prec];
        t.fn = lp.axis == kPlaneFwd ? xc.k->fwd : xc.k->inv;
        t.tm0 = &xc.tmx;
        t.tm1 = &xc.tmy;
        t.kc = xc.ctr.dev();
        t.blocks = xc.blocks;
        t.threads = xc.k->threads;
        t.smem = xc.k->smem;
        return true;
    }
    const ZCfg& zc = c->zpass[prec];
    if (lp.axis == 2 && zc.k && !c->ext && lp.red == RED_NONE && lp.store &&
        !lp.from_scratch && !lp.to_scratch && a.in == state_of(c, prec) &&
        lp.ops == std::vector<int>{OP_FFT_F, OP_KPHASE, OP_FFT_I}) {
        t.fn = zc.k->fn;
        t.tm0 = t.tm1 = &zc.tm;
        t.kc = zc.ctr.dev();
        t.blocks = zc.blocks;
        t.threads = zc.k->threads;
        t.smem = zc.k->smem;
        return true;
    }
    return false;
}

cudaError_t launch_tile(const TileLaunch& t, const PassArgs& a, cudaStream_t s, bool pdl) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(t.blocks);
    cfg.blockDim = dim3(t.threads);
    cfg.dynamicSmemBytes = t.smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    PassArgs pa = a;
    XYCounters kc = t.kc;
    void* args[] = {const_cast<CUtensorMap*>(t.tm0), const_cast<CUtensorMap*>(t.tm1), &pa, &kc};
    return cudaLaunchKernelExC(&cfg, t.fn, args);
}

gpue_status launch_pass(gpue_ctx* c, int prec, const LPass& lp, int gstate, bool pdl) {
    PassArgs a;
    gpue_status st = make_pass_args(c, prec, lp, gstate, a);
    if (st) return st;
    a.active = nullptr;  // a single solve always runs
    TileLaunch tl;
    if (tile_pass(c, prec, lp, a, tl)) {
        CK(launch_tile(tl, a, c->stream, pdl));
        c->launches++;
        return GPUE_OK;
    }
    if (lp.axis >= kPlaneFwd) {
        const PlaneCfg& pc = c->plane[prec];
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(pc.blocks);
        cfg.blockDim = dim3(pc.k->threads);
        cfg.dynamicSmemBytes = pc.k->smem;
        cfg.stream = c->stream;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = pc.k->cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = pdl ? 2 : 1;
        CK(cudaLaunchKernelEx(&cfg, lp.axis == kPlaneFwd ? pc.k->fwd : pc.k->inv, a));
        c->launches++;
        return GPUE_OK;
    }
    const LaunchCfg& lc = c->lc[prec][lp.axis];
    void (*fn)(PassArgs) = lp.axis == 0 ? (c->ext ? lc.k->row_ext : lc.k->row)
                                        : (c->ext ? lc.k->col_ext : lc.k->col);
    CK(launch_kernel(fn, lc.blocks, lc.threads, lc.smem, c->stream, pdl, a));
    c->launches++;
    return GPUE_OK;
}

// Logical passes of step i (see the file header).  guard: real-time norm
// guard period (0 off): steps with i % guard == guard-1 end with a NORM, and
// the factor is folded into the K pass of the next step (i % guard == 0).
void step_passes(gpue_ctx* c, int i, int gstate, bool scale_first, double rexp, int guard,
                 std::vector<LPass>& out, bool plane) {
    const bool g_norm = guard > 0 && i % guard == guard - 1;
    const bool g_apply = guard > 0 && i % guard == 0;
    const bool imag = gstate == 0;
    const double gdt = imag ? c->p.gdt * rexp : c->p.dt;
    const double tnow = (imag ? c->p.gdt : c->p.dt) * i;
    auto P = [&](int axis, std::vector<int> ops) {
        LPass lp;
        lp.axis = axis;
        lp.ops = ops;
        lp.gauge_dt = gdt;
        lp.time = tnow;
        return lp;
    };
    // gauge axes in GPUE's order for this step (x,y,z when i is odd, z,y,x
    // otherwise), leaving out axes whose factor is identically 1
    std::vector<int> gaxes;
    if (c->p.corotating) {
        const int order1[3] = {0, 1, 2}, order0[3] = {2, 1, 0};
        const int* ord = (i % 2) ? order1 : order0;
        for (int k = 0; k < 3; ++k)
            if (ord[k] < c->dim && axis_gauge_active(c, ord[k])) gaxes.push_back(ord[k]);
    }
    std::vector<LPass> s;
    if (plane && c->dim == 3 && gaxes.empty()) {
        // XY[scale V/2 Fx Fy] Z[Fz K Iz] XY[Ix Iy V/2]
        LPass f = P(kPlaneFwd, {});
        if (scale_first) f.ops.push_back(OP_SCALE);
        s.push_back(f);
        LPass kp = P(2, {OP_FFT_F, OP_KPHASE, OP_FFT_I});
        if (g_apply) kp.kscale_slot = kGuard;
        s.push_back(kp);
        s.push_back(P(kPlaneInv, {}));
    } else {
        std::vector<int> first;
        if (scale_first) first.push_back(OP_SCALE);
        first.push_back(OP_VHALF);
        first.push_back(OP_FFT_F);
        const int kaxis = c->dim == 3 ? 2 : 1;
        s.push_back(P(0, first));
        if (c->dim == 3) s.push_back(P(1, {OP_FFT_F}));
        LPass kp = P(kaxis, {OP_FFT_F, OP_KPHASE, OP_FFT_I});
        if (g_apply) kp.kscale_slot = kGuard;
        s.push_back(kp);
        if (c->dim == 3) s.push_back(P(1, {OP_FFT_I}));
        size_t g0 = 0;
        if (!gaxes.empty() && gaxes[0] == 0) {
            s.push_back(P(0, {OP_FFT_I, OP_VHALF, OP_FFT_F, OP_GAUGE, OP_FFT_I}));
            g0 = 1;
        } else {
            s.push_back(P(0, {OP_FFT_I, OP_VHALF}));
        }
        for (size_t k = g0; k < gaxes.size(); ++k) s.push_back(P(gaxes[k], {OP_FFT_F, OP_GAUGE, OP_FFT_I}));
    }
    if (imag || g_norm) {
        LPass& last = s.back();
        last.ops.push_back(OP_NORM);
        last.red = RED_NORM;
        last.red_slot = imag ? kScale : kGuard;
        last.red_target = imag ? kTargetImag : kTargetReal;
        last.red_blocks = imag;  // the guard factor is only read by the next K pass
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
            bool has_scale = false, q_gauge = false, p_gauge = false, p_red = false;
            for (int op : p.ops) has_scale |= (op == OP_SCALE), p_gauge |= (op == OP_GAUGE);
            for (int op : q.ops) q_gauge |= (op == OP_GAUGE);
            p_red = p.red != RED_NONE;
            const bool q_red_ok = q.red == RED_NONE || (!q.red_blocks && !p_red);
            if (q.axis == p.axis && q_red_ok && !has_scale && q.store && p.store &&
                !q.to_scratch && !p.from_scratch && !(q_gauge && p_gauge) &&
                q.kscale_slot < 0 && p.kscale_slot < 0 &&
                q.ops.size() + p.ops.size() <= (size_t)kMaxOps) {
                for (int op : p.ops) q.ops.push_back(op);
                if (p_red) {
                    q.red = p.red;
                    q.red_slot = p.red_slot;
                    q.red_target = p.red_target;
                    q.red_blocks = p.red_blocks;
                    q.ctr = p.ctr;
                }
                if (p_gauge) q.gauge_dt = p.gauge_dt;
                continue;
            }
        }
        o.push_back(p);
    }
    v.swap(o);
}

// Energy: kinetic sum K|psi_k|^2 via an unnormalised forward transform into
// scratch (divided by N on the host), and the real-space terms.
std::vector<LPass> energy_passes(const gpue_ctx* c, bool scale_pending) {
    std::vector<LPass> v;
    LPass x;
    x.axis = 0;
    if (scale_pending) x.ops.push_back(OP_SCALE);
    x.ops.push_back(OP_FFT_F);
    x.to_scratch = true;
    v.push_back(x);
    if (c->dim == 3) {
        LPass y;
        y.axis = 1;
        y.ops = {OP_FFT_F};
        y.from_scratch = true;
        v.push_back(y);
    }
    LPass last;
    last.axis = c->dim == 3 ? 2 : 1;
    last.ops = {OP_FFT_F, OP_EKIN};
    last.from_scratch = true;
    last.store = false;
    last.red = RED_SUM;
    last.red_slot = kEkin;
    last.ctr = kCtrEkin;
    v.push_back(last);
    return v;
}

EnergyArgs energy_args(gpue_ctx* c, int prec, bool scale_pending) {
    const Tables& tb = c->tab[prec];
    EnergyArgs e;
    std::memset(&e, 0, sizeof e);
    e.psi = state_of(c, prec);
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
    if (c->ext) {
        e.vtab = c->vtab;
        if (c->use_atab) {
            for (int i = 0; i < 3; ++i) e.atab[i] = c->atab[i];
            e.lterm = (c->p.corotating && c->dim > 1) ? 1 : 0;
        }
    }
    e.dx = c->ax[0].dx;
    e.dy = c->ax[1].dx;
    e.dz = c->ax[2].dx;
    e.hbar = c->p.hbar;
    e.red.kind = RED_SUM;
    e.red.partials = c->partials + (c->partials_cap - kAuxPartials);
    e.red.counter = c->counters + kCtrEreal;
    e.red.out = c->scal + kEreal;
    return e;
}

// after_pass: the energy passes follow a pass kernel in the stream
gpue_status launch_energy(gpue_ctx* c, int prec, int gstate, bool scale_pending,
                          bool after_pass = false) {
    bool pdl = after_pass;
    for (auto& lp : energy_passes(c, scale_pending)) {
        gpue_status st = launch_pass(c, prec, lp, gstate, pdl);
        if (st) return st;
        pdl = true;
    }
    EnergyArgs e = energy_args(c, prec, scale_pending);
    if (c->obs_out) {
        // the observables reduction in place of the real-space energy pass:
        // one read of psi, energy_calc's real-space sum left in kEreal
        ObsArgs oa;
        std::memset(&oa, 0, sizeof oa);
        oa.e = e;
        oa.partials = e.red.partials;
        oa.counter = e.red.counter;
        oa.out = c->obs_dev;
        oa.ereal = c->scal + kEreal;
        const int blocks = (int)std::min<long>(c->sms * 2, (kAuxPartials - kObsN) / kObsN);
        if (prec == GPUE_PREC_FP32) k_observables<float><<<blocks, 256, 0, c->stream>>>(oa);
        else k_observables<double><<<blocks, 256, 0, c->stream>>>(oa);
    } else {
        const int blocks = c->sms * 4;
        if (prec == GPUE_PREC_FP32) k_energy_real<float><<<blocks, 256, 0, c->stream>>>(e);
        else k_energy_real<double><<<blocks, 256, 0, c->stream>>>(e);
    }
    c->launches++;
    CK(cudaGetLastError());
    return GPUE_OK;
}

// The observables of the latest energy check (launch_energy with obs_out set)
// into the caller's array entry k, scaled as gpue_observables_get scales them.
gpue_status read_check_observables(gpue_ctx* c, int k) {
    if (!c->obs_out || k >= c->obs_cap) return GPUE_OK;
    double h[kObsN], ekin;
    CK(cudaMemcpyAsync(h, c->obs_dev, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&ekin, c->scal + kEkin, sizeof ekin, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    gpue_observables& o = c->obs_out[k];
    std::memset(&o, 0, sizeof o);
    const double dV = c->dV;
    o.norm = h[kObsNorm] * dV;
    o.e_kinetic = ekin / (double)c->N * dV;
    o.e_potential = h[kObsPot] * dV;
    o.e_interaction = h[kObsInt] * dV;
    o.e_rotation = h[kObsRot] * dV;
    o.energy = o.e_kinetic + o.e_potential + o.e_interaction + o.e_rotation;
    o.x = h[kObsX] * dV;
    o.y = h[kObsY] * dV;
    o.z = h[kObsZ] * dV;
    o.r2 = h[kObsR2] * dV;
    o.q = h[kObsQ] * dV;
    o.lz = h[kObsLz] * dV;
    return GPUE_OK;
}

gpue_status read_energy(gpue_ctx* c, double* E) {
    double h[kNScal];
    CK(cudaMemcpyAsync(h, c->scal, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *E = (h[kEkin] / (double)c->N + h[kEreal]) * c->dV;
    return GPUE_OK;
}

gpue_status scale_state(gpue_ctx* c, int prec, int slot) {
    void* psi = state_of(c, prec);
    if (prec == GPUE_PREC_FP32)
        k_scale<float><<<c->sms * 8, 256, 0, c->stream>>>(psi, c->N, c->scal + slot);
    else
        k_scale<double><<<c->sms * 8, 256, 0, c->stream>>>(psi, c->N, c->scal + slot);
    c->launches++;
    CK(cudaGetLastError());
    return GPUE_OK;
}

gpue_status apply_pending_scale(gpue_ctx* c, int prec) {
    if (!c->pending_scale) return GPUE_OK;
    gpue_status st = scale_state(c, prec, kScale);
    if (st) return st;
    c->pending_scale = false;
    return GPUE_OK;
}

// sum |psi|^2 of a state into a scalar slot (stream-ordered, no sync)
gpue_status norm_to_slot(gpue_ctx* c, int prec, int slot) {
    RedArgs r;
    std::memset(&r, 0, sizeof r);
    r.kind = RED_SUM;
    r.partials = c->partials + (c->partials_cap - kAuxPartials);
    r.counter = c->counters + kCtrMisc;
    r.out = c->scal + slot;
    void* psi = state_of(c, prec);
    if (prec == GPUE_PREC_FP32) k_norm<float><<<c->sms * 4, 256, 0, c->stream>>>(psi, c->N, r);
    else k_norm<double><<<c->sms * 4, 256, 0, c->stream>>>(psi, c->N, r);
    c->launches++;
    CK(cudaGetLastError());
    return GPUE_OK;
}

gpue_status norm_now(gpue_ctx* c, int prec, double* out) {
    gpue_status st = norm_to_slot(c, prec, kNorm);
    if (st) return st;
    double h;
    CK(cudaMemcpyAsync(&h, c->scal + kNorm, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *out = h * c->dV;
    return GPUE_OK;
}

// Enqueue steps [i0, i1) (+ energy passes after the last one when asked).
gpue_status enqueue_steps(gpue_ctx* c, int prec, int i0, int i1, int gstate, bool scale_first,
                          const std::vector<double>& rexp, bool energy_after, int guard) {
    std::vector<LPass> v;
    // every imaginary-time step after the first renormalises the state the
    // previous step left (the deferred parSum scale)
    const bool plane = plane_ok(c, prec);
    for (int i = i0; i < i1; ++i)
        step_passes(c, i, gstate, i == i0 ? scale_first : gstate == 0,
                    rexp.empty() ? 1.0 : rexp[i], guard, v, plane);
    if (!c->time_dep) fuse(v);  // fused passes would mix two steps' times
    for (size_t k = 0; k < v.size(); ++k) {
        gpue_status st = launch_pass(c, prec, v[k], gstate, k > 0);
        if (st) return st;
    }
    if (energy_after) {
        gpue_status st = launch_energy(c, prec, gstate, gstate == 0, !v.empty());
        if (st) return st;
    }
    return GPUE_OK;
}

gpue_status run_segment(gpue_ctx* c, int prec, int i0, int i1, int gstate, bool scale_first,
                        const std::vector<double>& rexp, bool energy_after, int guard) {
    // per-step arguments (ramp exponent, expression time) are not cached
    if (!rexp.empty() || c->time_dep)
        return enqueue_steps(c, prec, i0, i1, gstate, scale_first, rexp, energy_after, guard);
    // the pass pattern repeats with the gauge order (i % 2) and the guard period
    GraphKey key{prec, gstate, i0 % (guard == 4 ? 4 : 2), i1 - i0, scale_first ? 1 : 0,
                 energy_after ? 1 : 0, guard, c->obs_out ? 1 : 0};
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
        const long before = c->launches;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        gpue_status st =
            enqueue_steps(c, prec, i0, i1, gstate, scale_first, rexp, energy_after, guard);
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

// ------------------------------------------------------------- autotune --

// Device time of a few steps of this context's own schedule (the time kind
// its tables are built for), so a candidate launch shape is compared on the
// passes it will run, phases and reductions included.  The state and the
// scalar slots are saved first and put back after.
gpue_status time_steps(gpue_ctx* c, int prec, float* us) {
    const int gstate = c->tab[prec].built_for < 0 ? 0 : c->tab[prec].built_for;
    gpue_status st = build_tables(c, prec, gstate);
    if (st) return st;
    if (!c->have_wfc)  // any finite state times the same; this one is ~1e-2 (FP32)
        CK(cudaMemsetAsync(state_of(c, prec), 0x3C, c->N * elem_size(prec), c->stream));
    const int nsteps = 4, reps = 2;
    double saved[kNScal];
    const size_t bytes = c->N * elem_size(prec);
    CK(cudaMemcpyAsync(c->scratch, state_of(c, prec), bytes, cudaMemcpyDeviceToDevice,
                       c->stream));
    CK(cudaMemcpyAsync(saved, c->scal, sizeof saved, cudaMemcpyDeviceToHost, c->stream));
    const std::vector<double> rexp;
    const long launches = c->launches;
    st = enqueue_steps(c, prec, 0, nsteps, gstate, false, rexp, false, 0);
    if (st) return st;
    CK(cudaEventRecord(c->ev0, c->stream));
    for (int r = 0; r < reps && !st; ++r)
        st = enqueue_steps(c, prec, 0, nsteps, gstate, false, rexp, false, 0);
    if (st) return st;
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaMemcpyAsync(state_of(c, prec), c->scratch, bytes, cudaMemcpyDeviceToDevice,
                       c->stream));
    CK(cudaMemcpyAsync(c->scal, saved, sizeof saved, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->launches = launches;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *us = ms * 1e3f / (reps * nsteps);
    return GPUE_OK;
}

gpue_status autotune_ctx(gpue_ctx* c, int prec, bool force) {
    for (int axis = 0; axis < c->dim; ++axis) {
        TuneChoice tc;
        if (!force && cached_choice(c, prec, axis, tc)) {
            gpue_status st = plan_axis(c, prec, axis);
            if (st) return st;
            continue;
        }
        const PassKernel* ks[8];
        const int nk = find_pass_kernels(kprec(prec), c->ax[axis].n, ks, 8);
        if (!nk) return fail(c, GPUE_ERR_UNSUPPORTED, "no FFT plan for length %d", c->ax[axis].n);
        LaunchCfg def;
        if (!build_cfg(c, prec, axis, ks[0], default_lines(c, axis, ks[0]), def))
            return fail(c, GPUE_ERR_CUDA, "no launch shape for length %d", c->ax[axis].n);
        c->lc[prec][axis] = def;
        float def_us = 0.f;
        gpue_status st = time_steps(c, prec, &def_us);
        if (st) return st;
        LaunchCfg best = def;
        float best_us = def_us;
        for (int i = 0; i < nk; ++i) {
            for (int C = 1; C <= 64; C *= 2) {
                LaunchCfg cand;
                if (!build_cfg(c, prec, axis, ks[i], C, cand)) continue;
                if (cand.k == def.k && cand.lines == def.lines) continue;
                c->lc[prec][axis] = cand;
                float t0 = 0.f, t1 = 0.f;
                st = time_steps(c, prec, &t0);
                if (!st) st = time_steps(c, prec, &t1);
                if (st) return st;
                const float t = std::min(t0, t1);
                if (t < 0.97f * best_us) {  // a clear gain only: noise must not flip plans
                    best = cand;
                    best_us = t;
                }
            }
        }
        best.tuned = true;
        best.us = best_us;
        best.default_us = def_us;
        c->lc[prec][axis] = best;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[TuneKey{prec, c->dim, c->ax[axis].n, axis}] =
            TuneChoice{best.k->ra, best.k->rb, best.k->rc, best.k->p, best.lines, best_us, def_us};
    }
    destroy_graphs(c);  // the captured segments hold the old launch shapes
    return GPUE_OK;
}

struct LoopOut {
    int done = 0, early = 0, n_en = 0;
    double energy = NAN;
};

// The step loop of evolve() on the state of precision `prec`, absolute steps
// [off, off + nsteps), energy checks and early stop as GPUE does them.
// Mean device time of each pass of a step (gpue_time_passes).
gpue_status time_passes(gpue_ctx* c, int prec, int gstate, int nsteps, std::vector<float>& us,
                        std::vector<int>& kinds) {
    gpue_status st = build_tables(c, prec, gstate);
    if (st) return st;
    if (!c->have_wfc)  // any finite state times the same; this one is ~1e-2 (FP32)
        CK(cudaMemsetAsync(state_of(c, prec), 0x3C, c->N * elem_size(prec), c->stream));
    double saved[kNScal];
    const size_t bytes = c->N * elem_size(prec);
    CK(cudaMemcpyAsync(c->scratch, state_of(c, prec), bytes, cudaMemcpyDeviceToDevice,
                       c->stream));
    CK(cudaMemcpyAsync(saved, c->scal, sizeof saved, cudaMemcpyDeviceToHost, c->stream));
    const long launches = c->launches;
    const bool plane = plane_ok(c, prec);
    std::vector<std::vector<float>> per;  // [step][pass] ms
    std::vector<cudaEvent_t> ev;
    for (int i = 0; i < nsteps && !st; ++i) {
        std::vector<LPass> v;
        step_passes(c, i, gstate, i == 0 ? (gstate == 0 && c->pending_scale) : gstate == 0,
                    1.0, 0, v, plane);
        fuse(v);
        if (i == 0) {
            kinds.clear();
            for (const LPass& lp : v) kinds.push_back(lp.axis);
            ev.assign(v.size() + 1, nullptr);
            for (cudaEvent_t& e : ev)
                if (cudaEventCreate(&e) != cudaSuccess) st = GPUE_ERR_CUDA;
            if (st) break;
        }
        if (v.size() + 1 != ev.size()) break;  // a step of another shape: stop here
        std::vector<float> ms(v.size(), 0.f);
        if (cudaEventRecord(ev[0], c->stream) != cudaSuccess) st = GPUE_ERR_CUDA;
        for (size_t k = 0; k < v.size() && !st; ++k) {
            st = launch_pass(c, prec, v[k], gstate, false);
            if (!st && cudaEventRecord(ev[k + 1], c->stream) != cudaSuccess) st = GPUE_ERR_CUDA;
        }
        if (!st && cudaEventSynchronize(ev.back()) != cudaSuccess) st = GPUE_ERR_CUDA;
        for (size_t k = 0; k < v.size() && !st; ++k)
            if (cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]) != cudaSuccess) st = GPUE_ERR_CUDA;
        per.push_back(ms);
    }
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    c->launches = launches;
    // the state and the scalars as they were, whatever happened above
    CK(cudaMemcpyAsync(state_of(c, prec), c->scratch, bytes, cudaMemcpyDeviceToDevice,
                       c->stream));
    CK(cudaMemcpyAsync(c->scal, saved, sizeof saved, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (st) return fail(c, st, "gpue_time_passes: a launch or an event failed");
    us.assign(kinds.size(), 0.f);
    for (const auto& ms : per)
        for (size_t k = 0; k < ms.size() && k < us.size(); ++k) us[k] += ms[k] * 1e3f / per.size();
    return GPUE_OK;
}

gpue_status step_loop(gpue_ctx* c, int prec, int off, int nsteps, int gstate,
                      const gpue_evolve_opts& o, int guard, LoopOut& lo) {
    const int last = off + nsteps;
    std::vector<double> rexp;
    // ramp (src/evolution.cu:409-427): GPUE raises the gauge tables to
    // omega_0 every step, so the exponent at step i is cumulative
    if (c->p.ramp && gstate == 0 && c->p.corotating &&
        (axis_gauge_active(c, 0) || axis_gauge_active(c, 1) || axis_gauge_active(c, 2))) {
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
    // GPUE compares with the energy stored by the previous check
    // (par.dval("energy")), which a sliced run carries across calls
    double old_energy = off > 0 ? c->last_energy : 0.0;
    int i = off;
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
        gpue_status st = run_segment(c, prec, i, seg_end, gstate, scale_next, rexp, check, guard);
        if (st) return st;
        if (gstate == 0) {
            scale_next = true;
            c->pending_scale = true;
        }
        i = seg_end;
        lo.done = i - off;
        if (check) {
            double energy;
            st = read_energy(c, &energy);
            if (!st) st = read_check_observables(c, lo.n_en);
            if (st) return st;
            lo.energy = energy;
            lo.n_en++;
            c->last_energy = energy;
            const int step = i - 1;
            const bool stop =
                o.threshold_abs ? std::fabs(old_energy - energy) < o.energy_calc_threshold
                                : std::fabs(old_energy - energy) < o.energy_calc_threshold * old_energy;
            if (step != 0 && stop && gstate == 0) {
                lo.early = 1;
                break;
            }
            old_energy = energy;
        }
    }
    return GPUE_OK;
}

size_t ctx_bytes_estimate(int dim, int n, int prec) {
    auto al = [](size_t b) { return ((b + 255) / 256) * 256; };
    const size_t N = (size_t)n * n * (dim == 3 ? n : 1);
    const size_t cap = N / n + kAuxPartials + 1024;  // partials_cap (gpue_ctx_create)
    size_t b = al(N * elem_size(prec)) + al(N * 16);  // state, scratch
    b += al(kNScal * sizeof(double)) + al(cap * sizeof(double2)) +
         al(kNCtr * sizeof(unsigned)) + al(4 * sizeof(int));
    const size_t tn = 3 * (2 * al((size_t)n * 16) + al((size_t)n * 16) +
                           3 * al((size_t)n * 8));
    return b + tn;  // one precision's operator tables
}

size_t ctx_device_bytes(const gpue_ctx* c) {
    auto al = [](size_t b) { return ((b + 255) / 256) * 256; };
    size_t b = ctx_bytes_estimate(c->dim, c->ax[0].n, c->prec);
    if (c->psi64) b += al(c->N * 16);  // FP64 shadow
    if (c->tab[1 - c->prec].buf) {  // the other precision's tables (polishing)
        for (int a = 0; a < 3; ++a) {
            const size_t n = c->ax[a].n;
            b += 3 * al(n * 16) + 3 * al(n * 8);
        }
    }
    if (c->vtab) b += al(c->N * 8);
    for (auto t : c->atab)
        if (t) b += al(c->N * 8);
    return b;
}

gpue_status ensure_shadow(gpue_ctx* c) {
    if (c->psi64) return GPUE_OK;
    CK(cudaMalloc(&c->psi64, c->N * 16));
    for (int a = 0; a < c->dim; ++a) {
        gpue_status st = plan_axis(c, GPUE_PREC_FP64, a);
        if (st) return st;
    }
    return GPUE_OK;
}

// After a polish the FP64 shadow holds the state; bring it back.
gpue_status unpolish(gpue_ctx* c) {
    if (!c->polished) return GPUE_OK;
    k_convert<double, float><<<c->sms * 8, 256, 0, c->stream>>>(c->psi64, c->psi, c->N);
    CK(cudaGetLastError());
    c->polished = false;
    return GPUE_OK;
}

}  // namespace gpue_eng

namespace gpue_eng {

// Uploads full-field V and A tables (FP64, N each); the passes then use the
// table forms (ext kernels) and, when use_a, the tabulated gauge.
gpue_status install_fields(gpue_ctx* c, const std::vector<double>& V,
                           const std::vector<double> (&A)[3], bool use_a) {
    if (!c->vtab) {
        CK(cudaMalloc(&c->vtab, c->N * sizeof(double)));
        for (auto& t : c->atab) CK(cudaMalloc(&t, c->N * sizeof(double)));
    }
    CK(cudaMemcpy(c->vtab, V.data(), c->N * sizeof(double), cudaMemcpyHostToDevice));
    for (int a = 0; a < 3; ++a) {
        CK(cudaMemcpy(c->atab[a], A[a].data(), c->N * sizeof(double), cudaMemcpyHostToDevice));
        bool nz_any = false;
        for (double v : A[a]) nz_any |= (v != 0.0);
        c->atab_nonzero[a] = nz_any;
    }
    c->use_atab = use_a;
    return GPUE_OK;
}

}  // namespace gpue_eng

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
    const double Rxy =
        std::pow(15.0, 0.2) * std::pow(N * a_s * std::sqrt(mass * p->omegaZ / HBAR), 0.2);
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
    if (c->dim != 2 && c->dim != 3) return GPUE_ERR_INVALID_ARG;
    const int nx = p->xDim, ny = p->yDim, nz = c->dim == 3 ? p->zDim : 1;
    if (nx < 2 || ny != nx || (c->dim == 3 && nz != nx)) return GPUE_ERR_INVALID_ARG;
    if (!(p->xMax > 0) || !(p->hbar > 0) || !(p->mass > 0)) return GPUE_ERR_INVALID_ARG;
    if (c->dim > 1 && !(p->yMax > 0)) return GPUE_ERR_INVALID_ARG;
    if (c->dim > 2 && !(p->zMax > 0)) return GPUE_ERR_INVALID_ARG;
    if (!gpue_supported_length(c->prec, nx)) return GPUE_ERR_UNSUPPORTED;
    build_axis(c->ax[0], nx, p->xMax, true);
    build_axis(c->ax[1], ny, p->yMax, true);
    build_axis(c->ax[2], nz, p->zMax, c->dim == 3);
    c->N = (long)nx * ny * nz;
    c->dV = c->ax[0].dx * c->ax[1].dx * (c->dim == 3 ? c->ax[2].dx : 1.0);
    c->device = p->device;
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    CK(cudaMalloc(&c->psi, c->N * elem_size(c->prec)));
    CK(cudaMalloc(&c->scratch, c->N * 16));
    CK(cudaMalloc(&c->scal, kNScal * sizeof(double)));
    c->partials_cap = c->N / nx + kAuxPartials + 1024;
    CK(cudaMalloc(&c->partials, c->partials_cap * sizeof(double2)));
    CK(cudaMalloc(&c->counters, kNCtr * sizeof(unsigned)));
    CK(cudaMalloc(&c->dflags, 4 * sizeof(int)));
    CK(cudaMemsetAsync(c->dflags, 0, 4 * sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->counters, 0, kNCtr * sizeof(unsigned), c->stream));
    double hs[kNScal] = {1.0, 0.0, 0.0, 0.0, 1.0, 1.0 / c->dV, 1.0, 1.0};
    CK(cudaMemcpyAsync(c->scal, hs, sizeof hs, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->psi, 0, c->N * elem_size(c->prec), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    gpue_status st = build_tables(c, c->prec, 0);
    if (st) return st;
    for (int a = 0; a < c->dim; ++a) {
        st = plan_axis(c, c->prec, a);
        if (st) return st;
    }
    st = plan_plane(c, c->prec);
    if (!st) st = plan_zpass(c, c->prec);
    if (!st) st = plan_xy(c, c->prec);
    if (st) return st;
    const char* tune = std::getenv("GPUE_AUTOTUNE");
    if (tune && tune[0] == '1') {
        st = autotune_ctx(c, c->prec, false);
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
    if (c->psi64) cudaFree(c->psi64);
    for (auto& x : c->xy)
        if (x.ctr.mem) cudaFree(x.ctr.mem);
    for (auto& z : c->zpass)
        if (z.ctr.mem) cudaFree(z.ctr.mem);
    if (c->vtab) cudaFree(c->vtab);
    for (auto t : c->atab)
        if (t) cudaFree(t);
    if (c->progs) cudaFree(c->progs);
    if (c->vtx_ws) cudaFree(c->vtx_ws);
    if (c->obs_dev) cudaFree(c->obs_dev);
    cudaFree(c->scratch);
    cudaFree(c->scal);
    cudaFree(c->partials);
    cudaFree(c->counters);
    cudaFree(c->dflags);
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
    const cudaMemcpyKind kind =
        mem == GPUE_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (dtype == want) {
        CK(cudaMemcpyAsync(c->psi, psi, in_bytes, kind, c->stream));
    } else {
        CK(cudaMemcpyAsync(c->scratch, psi, in_bytes, kind, c->stream));
        if (dtype == GPUE_C128)
            k_convert<double, float><<<c->sms * 8, 256, 0, c->stream>>>(c->scratch, c->psi, c->N);
        else
            k_convert<float, double><<<c->sms * 8, 256, 0, c->stream>>>(c->scratch, c->psi, c->N);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(c->stream));
    c->have_wfc = true;
    c->pending_scale = false;
    c->polished = false;
    return GPUE_OK;
}

gpue_status gpue_get_wfc(gpue_ctx* c, void* psi, int32_t mem, int32_t dtype) {
    if (!c || !psi || (mem != GPUE_MEM_HOST && mem != GPUE_MEM_DEVICE) ||
        (dtype != GPUE_C128 && dtype != GPUE_C64))
        return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    const int sp = c->polished ? GPUE_PREC_FP64 : c->prec;
    gpue_status st = apply_pending_scale(c, sp);
    if (st) return st;
    void* src = state_of(c, sp);
    const int have = sp == GPUE_PREC_FP32 ? GPUE_C64 : GPUE_C128;
    const size_t out_bytes = c->N * (dtype == GPUE_C128 ? 16 : 8);
    const cudaMemcpyKind kind =
        mem == GPUE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (dtype == have) {
        CK(cudaMemcpyAsync(psi, src, out_bytes, kind, c->stream));
    } else {
        if (have == GPUE_C64)
            k_convert<float, double><<<c->sms * 8, 256, 0, c->stream>>>(src, c->scratch, c->N);
        else
            k_convert<double, float><<<c->sms * 8, 256, 0, c->stream>>>(src, c->scratch, c->N);
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
    const int sp = c->polished ? GPUE_PREC_FP64 : c->prec;
    const int gs = c->tab[sp].built_for < 0 ? 0 : c->tab[sp].built_for;
    gpue_status st = build_tables(c, sp, gs);
    if (st) return st;
    st = launch_energy(c, sp, gs, c->pending_scale);
    if (st) return st;
    return read_energy(c, E);
}

gpue_status gpue_observables_get(gpue_ctx* c, gpue_observables* o) {
    if (!c || !o) return GPUE_ERR_INVALID_ARG;
    if (!c->have_wfc) return fail(c, GPUE_ERR_STATE, "no wavefunction set");
    CK(cudaSetDevice(c->device));
    const int sp = c->polished ? GPUE_PREC_FP64 : c->prec;
    const int gs = c->tab[sp].built_for < 0 ? 0 : c->tab[sp].built_for;
    gpue_status st = build_tables(c, sp, gs);
    if (st) return st;
    bool pdl = false;
    for (auto& lp : energy_passes(c, c->pending_scale)) {
        st = launch_pass(c, sp, lp, gs, pdl);
        if (st) return st;
        pdl = true;
    }
    ObsArgs oa;
    std::memset(&oa, 0, sizeof oa);
    oa.e = energy_args(c, sp, c->pending_scale);
    double2* aux = c->partials + (c->partials_cap - kAuxPartials);
    const int blocks = (int)std::min<long>(c->sms * 2, (kAuxPartials - kObsN) / kObsN);
    oa.partials = aux;
    oa.counter = c->counters + kCtrMisc;
    oa.out = reinterpret_cast<double*>(aux + (long)kObsN * blocks);
    if (sp == GPUE_PREC_FP32) k_observables<float><<<blocks, 256, 0, c->stream>>>(oa);
    else k_observables<double><<<blocks, 256, 0, c->stream>>>(oa);
    c->launches++;
    CK(cudaGetLastError());
    double h[kObsN], ekin;
    CK(cudaMemcpyAsync(h, oa.out, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&ekin, c->scal + kEkin, sizeof ekin, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memset(o, 0, sizeof *o);
    const double dV = c->dV;
    o->norm = h[kObsNorm] * dV;
    o->e_kinetic = ekin / (double)c->N * dV;
    o->e_potential = h[kObsPot] * dV;
    o->e_interaction = h[kObsInt] * dV;
    o->e_rotation = h[kObsRot] * dV;
    o->energy = o->e_kinetic + o->e_potential + o->e_interaction + o->e_rotation;
    o->x = h[kObsX] * dV;
    o->y = h[kObsY] * dV;
    o->z = h[kObsZ] * dV;
    o->r2 = h[kObsR2] * dV;
    o->q = h[kObsQ] * dV;
    o->lz = h[kObsLz] * dV;
    return GPUE_OK;
}

gpue_status gpue_set_check_observables(gpue_ctx* c, gpue_observables* out, int32_t cap) {
    if (!c || cap < 0 || (cap > 0 && !out)) return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (cap > 0 && !c->obs_dev) CK(cudaMalloc(&c->obs_dev, kObsN * sizeof(double)));
    c->obs_out = cap > 0 ? out : nullptr;
    c->obs_cap = cap;
    destroy_graphs(c);  // captured checks hold the other reduction
    return GPUE_OK;
}

gpue_status gpue_norm(gpue_ctx* c, double* out) {
    if (!c || !out) return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    const int sp = c->polished ? GPUE_PREC_FP64 : c->prec;
    gpue_status st = apply_pending_scale(c, sp);
    if (st) return st;
    return norm_now(c, sp, out);
}

gpue_status gpue_ctx_stream(gpue_ctx* c, void** s) {
    if (!c || !s) return GPUE_ERR_INVALID_ARG;
    *s = (void*)c->stream;
    return GPUE_OK;
}

// The Grid doubles an expression may name (parseArgs and init() store them).
static std::map<std::string, double> grid_doubles(const gpue_ctx* c, const char* const* names,
                                                  const double* values, int32_t n) {
    const gpue_params& p = c->p;
    std::map<std::string, double> m = {
        {"omega", p.omega},       {"gammaY", p.gammaY},       {"gdt", p.gdt},
        {"dt", p.dt},             {"omegaX", p.omegaX},       {"omegaY", p.omegaY},
        {"omegaZ", p.omegaZ},     {"interaction", p.interaction},
        {"x0_shift", p.x0_shift}, {"y0_shift", p.y0_shift},   {"z0_shift", p.z0_shift},
        {"mass", p.mass},         {"gDenConst", p.gDenConst}, {"xMax", p.xMax},
        {"yMax", p.yMax},         {"zMax", p.zMax},           {"dx", c->ax[0].dx},
        {"dy", c->ax[1].dx},      {"dz", c->dim == 3 ? c->ax[2].dx : 1.0},
        {"fudge", 0.0}};
    for (int a = 0; a < 3; ++a) {
        const char* nm[3][2] = {{"dpx", "pxMax"}, {"dpy", "pyMax"}, {"dpz", "pzMax"}};
        const double xm = a == 0 ? p.xMax : a == 1 ? p.yMax : p.zMax;
        const int na = a == 0 ? p.xDim : a == 1 ? p.yDim : p.zDim;
        if (xm > 0) {
            m[nm[a][0]] = kPI / xm;
            m[nm[a][1]] = (kPI / xm) * (na >> 1);
        }
    }
    for (int i = 0; i < n; ++i)
        if (names && names[i] && values) m[names[i]] = values[i];
    return m;
}

gpue_status gpue_load_param_text(gpue_ctx* c, const char* text, int32_t time_mode,
                                 const char* const* names, const double* values,
                                 int32_t nvalues) {
    if (!c || !text || (time_mode != 0 && time_mode != 1) || nvalues < 0)
        return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    std::map<std::string, AstExpr> ex;
    std::vector<std::string> order;
    std::string err;
    if (!ast_parse_file(text, grid_doubles(c, names, values, nvalues), ex, order, err))
        return fail(c, GPUE_ERR_AST, "%s", err.c_str());
    const gpue_params& p = c->p;
    const int nx = c->ax[0].n, ny = c->ax[1].n;
    const double dx = c->ax[0].dx, dy = c->ax[1].dx, dz = c->dim == 3 ? c->ax[2].dx : 1.0;
    const double zmax = c->dim == 3 ? p.zMax : 0.0;
    auto has = [&](const char* k) { return ex.count(k) > 0; };
    // static fields at t = 0 (find_field, src/dynamic.cu:605-616; generate_gauge
    // and generate_fields, src/operators.cu:472-618, 808-830)
    std::vector<double> V(c->N), A[3];
    for (auto& v : A) v.assign(c->N, 0.0);
    double axc, ayc;
    gauge_coefs(c, axc, ayc);
    const bool any_a = has("Ax") || has("Ay") || has("Az");
    const char* an[3] = {"Ax", "Ay", "Az"};
    for (long g = 0; g < c->N; ++g) {
        const int i = (int)(g % nx), j = (int)((g / nx) % ny), k = (int)(g / ((long)nx * ny));
        const double fx = dx * i - p.xMax, fy = dy * j - p.yMax, fz = dz * k - zmax;
        for (int a = 0; a < 3; ++a) {
            if (has(an[a])) A[a][g] = ast_eval_host(ex[an[a]], fx, fy, fz, 0.0);
            else if (a == 0) A[a][g] = -c->ax[1].x[j] * p.omega * p.omegaX * (axc != 0.0);
            else if (a == 1) A[a][g] = c->ax[0].x[i] * p.omega * p.omegaY * (ayc != 0.0);
        }
        if (has("V")) {
            V[g] = ast_eval_host(ex["V"], fx, fy, fz, 0.0);
        } else {
            const double vx = p.omegaX * (c->ax[0].x[i] + p.x0_shift);
            const double vy = p.gammaY * p.omegaY * (c->ax[1].x[j] + p.y0_shift);
            const double vz = (c->dim == 3 ? p.omegaZ : 0.0) *
                              (c->ax[2].x[k] + (c->dim == 3 ? p.z0_shift : 0.0));
            V[g] = 0.5 * p.mass * ((vx * vx + vy * vy + vz * vz) +
                                   (A[0][g] * A[0][g] + A[1][g] * A[1][g] + A[2][g] * A[2][g]));
        }
    }
    gpue_status st = install_fields(c, V, A, any_a);
    if (st) return st;
    // time-dependent expressions: evolve()'s *_time branches
    std::vector<AstInstr> progs;
    const char* pn[5] = {"V", "k", "Ax", "Ay", "Az"};
    c->time_dep = false;
    for (int k = 0; k < 5; ++k) {
        c->prog_off[k] = -1;
        c->prog_len[k] = 0;
        if (time_mode == 1 && has(pn[k]) && ex[pn[k]].time_dependent) {
            c->prog_off[k] = (int)progs.size();
            c->prog_len[k] = (int)ex[pn[k]].program.size();
            for (auto& in : ex[pn[k]].program) progs.push_back(in);
            c->time_dep = true;
        }
    }
    if (c->progs) {
        cudaFree(c->progs);
        c->progs = nullptr;
    }
    if (!progs.empty()) {
        CK(cudaMalloc(&c->progs, progs.size() * sizeof(AstInstr)));
        CK(cudaMemcpy(c->progs, progs.data(), progs.size() * sizeof(AstInstr),
                      cudaMemcpyHostToDevice));
    }
    c->ext = true;
    destroy_graphs(c);
    return GPUE_OK;
}

gpue_status gpue_set_gauge_tables(gpue_ctx* c, const double* Ax, const double* Ay,
                                  const double* Az) {
    if (!c || (!Ax && !Ay && !Az)) return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    const gpue_params& p = c->p;
    const int nx = c->ax[0].n, ny = c->ax[1].n;
    std::vector<double> V(c->N), A[3];
    const double* src[3] = {Ax, Ay, c->dim == 3 ? Az : nullptr};
    for (int a = 0; a < 3; ++a) {
        A[a].assign(c->N, 0.0);
        if (src[a]) std::copy(src[a], src[a] + c->N, A[a].begin());
    }
    // kharmonic_V (src/operators.cu:994-1008) with the tabulated A
    for (long g = 0; g < c->N; ++g) {
        const int i = (int)(g % nx), j = (int)((g / nx) % ny), k = (int)(g / ((long)nx * ny));
        const double vx = p.omegaX * (c->ax[0].x[i] + p.x0_shift);
        const double vy = p.gammaY * p.omegaY * (c->ax[1].x[j] + p.y0_shift);
        const double vz = (c->dim == 3 ? p.omegaZ : 0.0) *
                          (c->ax[2].x[k] + (c->dim == 3 ? p.z0_shift : 0.0));
        V[g] = 0.5 * p.mass * ((vx * vx + vy * vy + vz * vz) +
                               (A[0][g] * A[0][g] + A[1][g] * A[1][g] + A[2][g] * A[2][g]));
    }
    gpue_status st = install_fields(c, V, A, true);
    if (st) return st;
    for (int k = 0; k < 5; ++k) {
        c->prog_off[k] = -1;
        c->prog_len[k] = 0;
    }
    c->time_dep = false;
    c->ext = true;
    destroy_graphs(c);
    return GPUE_OK;
}

gpue_status gpue_set_potential_table(gpue_ctx* c, const double* V) {
    if (!c || !V) return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    if (!c->vtab) {
        CK(cudaMalloc(&c->vtab, c->N * sizeof(double)));
        for (auto& t : c->atab) {
            CK(cudaMalloc(&t, c->N * sizeof(double)));
            CK(cudaMemset(t, 0, c->N * sizeof(double)));
        }
        for (bool& nz : c->atab_nonzero) nz = false;
        c->use_atab = false;
    }
    CK(cudaMemcpy(c->vtab, V, c->N * sizeof(double), cudaMemcpyHostToDevice));
    // the table replaces a parameter-file V expression
    c->prog_off[0] = -1;
    c->prog_len[0] = 0;
    c->time_dep = false;
    for (int k = 1; k < 5; ++k) c->time_dep |= c->prog_len[k] > 0;
    c->ext = true;
    destroy_graphs(c);
    return GPUE_OK;
}

gpue_status gpue_ast_parse(const char* expr, const char* const* names, const double* values,
                           int32_t nvalues, void* nodes_out, int32_t cap, int32_t* count) {
    if (!expr || !count || cap < 0 || nvalues < 0) return GPUE_ERR_INVALID_ARG;
    std::map<std::string, double> m;
    for (int i = 0; i < nvalues; ++i)
        if (names && names[i] && values) m[names[i]] = values[i];
    std::string s;
    for (const char* q = expr; *q; ++q)
        if (!std::isspace((unsigned char)*q)) s.push_back(*q);
    AstExpr e;
    std::string err;
    if (!ast_parse(s, m, e, err)) return GPUE_ERR_AST;
    *count = (int32_t)e.nodes.size();
    if (nodes_out && cap >= *count) std::memcpy(nodes_out, e.nodes.data(), e.nodes.size() * sizeof(AstNode));
    else if (nodes_out) return GPUE_ERR_INVALID_ARG;
    return GPUE_OK;
}

gpue_status gpue_ast_parse_file(const char* text, const char* const* names,
                                const double* values, int32_t nvalues, int32_t entry,
                                char* name, int32_t name_cap, int32_t* time_flag,
                                void* nodes_out, int32_t cap, int32_t* count,
                                int32_t* nentries) {
    if (!text || !count || !nentries || cap < 0 || nvalues < 0 || entry < 0)
        return GPUE_ERR_INVALID_ARG;
    std::map<std::string, double> m;
    for (int i = 0; i < nvalues; ++i)
        if (names && names[i] && values) m[names[i]] = values[i];
    std::map<std::string, AstExpr> asts;
    std::vector<std::string> order;
    std::string err;
    if (!ast_parse_file(text, m, asts, order, err)) return GPUE_ERR_AST;
    *nentries = (int32_t)order.size();
    if (entry >= (int32_t)order.size()) return GPUE_ERR_INVALID_ARG;
    const std::string& nm = order[entry];
    const AstExpr& e = asts[nm];
    *count = (int32_t)e.nodes.size();
    if (time_flag) *time_flag = e.time_dependent ? 1 : 0;
    if (name) {
        if (name_cap <= (int32_t)nm.size()) return GPUE_ERR_INVALID_ARG;
        std::memcpy(name, nm.c_str(), nm.size() + 1);
    }
    if (nodes_out && cap >= *count)
        std::memcpy(nodes_out, e.nodes.data(), e.nodes.size() * sizeof(AstNode));
    else if (nodes_out)
        return GPUE_ERR_INVALID_ARG;
    return GPUE_OK;
}

gpue_status gpue_ctx_wfc_device(gpue_ctx* c, void** psi, int32_t* dtype) {
    if (!c || !psi || !dtype) return GPUE_ERR_INVALID_ARG;
    *psi = c->psi;
    *dtype = c->prec == GPUE_PREC_FP32 ? GPUE_C64 : GPUE_C128;
    return GPUE_OK;
}

gpue_status gpue_autotune(gpue_ctx* c, int32_t flags) {
    if (!c || (flags & ~1)) return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    return autotune_ctx(c, c->prec, (flags & 1) != 0);
}

gpue_status gpue_time_passes(gpue_ctx* c, int32_t gstate, int32_t nsteps, float* us,
                             int32_t* kinds, int32_t cap, int32_t* npass) {
    if (!c || !npass || nsteps < 1 || cap < 0 || (cap > 0 && (!us || !kinds)) ||
        (gstate != 0 && gstate != 1))
        return GPUE_ERR_INVALID_ARG;
    std::vector<float> t;
    std::vector<int> k;
    gpue_status st = time_passes(c, c->prec, gstate, nsteps, t, k);
    if (st) return st;
    *npass = (int32_t)t.size();
    for (int i = 0; i < cap && i < (int)t.size(); ++i) {
        us[i] = t[i];
        kinds[i] = k[i];
    }
    return GPUE_OK;
}

gpue_status gpue_get_plan(gpue_ctx* c, int32_t axis, gpue_plan_info* out) {
    if (!c || !out || axis < 0 || axis >= c->dim) return GPUE_ERR_INVALID_ARG;
    const LaunchCfg& lc = c->lc[c->prec][axis];
    if (!lc.k) return fail(c, GPUE_ERR_STATE, "axis %d not planned", axis);
    std::memset(out, 0, sizeof *out);
    out->n = lc.k->n;
    out->ra = lc.k->ra;
    out->rb = lc.k->rb;
    out->rc = lc.k->rc;
    out->threads_per_line = lc.k->p;
    out->lines_per_cta = lc.lines;
    out->threads = lc.threads;
    out->blocks = lc.blocks;
    out->tuned = lc.tuned ? 1 : 0;
    out->us = lc.us;
    out->default_us = lc.default_us;
    return GPUE_OK;
}

gpue_status gpue_list_plans(int32_t precision, int32_t n, gpue_plan_info* out, int32_t cap,
                            int32_t* count) {
    if (!count || cap < 0 || (cap > 0 && !out) ||
        (precision != GPUE_PREC_FP32 && precision != GPUE_PREC_FP64))
        return GPUE_ERR_INVALID_ARG;
    const PassKernel* ks[8];
    const int nk = find_pass_kernels(kprec(precision), n, ks, 8);
    *count = nk;
    for (int i = 0; i < nk && i < cap; ++i) {
        std::memset(&out[i], 0, sizeof out[i]);
        out[i].n = ks[i]->n;
        out[i].ra = ks[i]->ra;
        out[i].rb = ks[i]->rb;
        out[i].rc = ks[i]->rc;
        out[i].threads_per_line = ks[i]->p;
    }
    return GPUE_OK;
}

gpue_status gpue_set_plan(gpue_ctx* c, int32_t axis, int32_t ra, int32_t rb, int32_t rc,
                          int32_t p, int32_t lines) {
    if (!c || axis < 0 || axis >= c->dim || lines < 0) return GPUE_ERR_INVALID_ARG;
    CK(cudaSetDevice(c->device));
    const int prec = c->prec;
    const PassKernel* ks[8];
    const int nk = find_pass_kernels(kprec(prec), c->ax[axis].n, ks, 8);
    for (int i = 0; i < nk; ++i) {
        const PassKernel* k = ks[i];
        if (k->ra != ra || k->rb != rb || k->rc != rc || k->p != p) continue;
        LaunchCfg lc;
        if (!build_cfg(c, prec, axis, k, lines ? lines : default_lines(c, axis, k), lc))
            return fail(c, GPUE_ERR_INVALID_ARG, "plan (%d,%d,%d) P=%d: %d lines per CTA do not fit",
                        ra, rb, rc, p, lines);
        c->lc[prec][axis] = lc;
        destroy_graphs(c);
        return GPUE_OK;
    }
    return fail(c, GPUE_ERR_INVALID_ARG, "no compiled plan (%d,%d,%d) P=%d for length %d", ra,
                rb, rc, p, c->ax[axis].n);
}

gpue_status gpue_evolve(gpue_ctx* c, int32_t nsteps, int32_t gstate,
                        const gpue_evolve_opts* opts, gpue_evolve_result* res) {
    if (!c || nsteps < 0 || (gstate != 0 && gstate != 1)) return GPUE_ERR_INVALID_ARG;
    if (!c->have_wfc) return fail(c, GPUE_ERR_STATE, "no wavefunction set");
    CK(cudaSetDevice(c->device));
    gpue_evolve_opts o;
    std::memset(&o, 0, sizeof o);
    o.norm_guard = -1;
    if (opts) o = *opts;
    if (o.polish_steps < 0 || o.graph_chunk < 0 || o.step_offset < 0 ||
        (o.norm_guard_period != 0 && o.norm_guard_period != 1 && o.norm_guard_period != 2 &&
         o.norm_guard_period != 4))
        return GPUE_ERR_INVALID_ARG;
    if (o.no_sync && o.energy_calc_steps > 0)
        return fail(c, GPUE_ERR_INVALID_ARG, "no_sync excludes energy checks");
    const bool polish = o.polish_steps > 0 && c->prec == GPUE_PREC_FP32 && gstate == 0;
    // the guard assumes a unitary real-time step; GPUE's time-dependent gauge
    // multiplies by the raw A value, which is not, so the automatic choice
    // leaves it off then
    const bool unitary = c->prog_off[2] < 0 && c->prog_off[3] < 0 && c->prog_off[4] < 0;
    const bool guard_on = gstate == 1 && (o.norm_guard == 1 ||
                                          (o.norm_guard < 0 && c->prec == GPUE_PREC_FP32 &&
                                           unitary));
    // every second step by default: the same FP32 energy error as every step
    // (4e-7 over 20000 steps of the 1024^2 rotating case), 4 % less time
    const int guard = guard_on ? (o.norm_guard_period > 0 ? o.norm_guard_period : 2) : 0;
    gpue_status st = unpolish(c);
    if (st) return st;
    st = build_tables(c, c->prec, gstate);
    if (st) return st;
    c->launches = 0;
    const int off = o.step_offset;
    CK(cudaEventRecord(c->ev0, c->stream));
    if (guard) {
        st = norm_to_slot(c, c->prec, kTargetReal);
        if (st) return st;
        CK(cudaMemcpyAsync(c->scal + kGuard, c->scal + kOne, sizeof(double),
                           cudaMemcpyDeviceToDevice, c->stream));
    }
    LoopOut lo;
    st = step_loop(c, c->prec, off, nsteps, gstate, o, guard, lo);
    if (st) return st;
    st = apply_pending_scale(c, c->prec);
    if (st) return st;
    // a guard factor computed by the last step has not been applied yet
    const int last = off + lo.done - 1;
    if (guard && lo.done > 0 && last % guard == guard - 1) {
        st = scale_state(c, c->prec, kGuard);
        if (st) return st;
    }
    if (polish) {
        // FP64 polishing steps that continue the imaginary-time run
        st = ensure_shadow(c);
        if (st) return st;
        st = build_tables(c, GPUE_PREC_FP64, 0);
        if (st) return st;
        k_convert<float, double><<<c->sms * 8, 256, 0, c->stream>>>(c->psi, c->psi64, c->N);
        CK(cudaGetLastError());
        gpue_evolve_opts po = o;
        po.energy_calc_steps = 0;
        LoopOut pl;
        st = step_loop(c, GPUE_PREC_FP64, off + lo.done, o.polish_steps, 0, po, 0, pl);
        if (st) return st;
        st = apply_pending_scale(c, GPUE_PREC_FP64);
        if (st) return st;
        c->polished = true;
        lo.done += pl.done;
    }
    if (o.no_sync) {
        if (res) {
            std::memset(res, 0, sizeof *res);
            res->steps_done = lo.done;
            res->energy = NAN;
            res->kernel_launches = c->launches;
        }
        return GPUE_OK;
    }
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (c->plane[c->prec].k || c->xy[c->prec].k || c->zpass[c->prec].k) {
        int gave_up = 0;
        CK(cudaMemcpy(&gave_up, c->dflags + 3, sizeof gave_up, cudaMemcpyDeviceToHost));
        if (gave_up) {
            CK(cudaMemset(c->dflags + 3, 0, sizeof gave_up));
            return fail(c, GPUE_ERR_TIMEOUT, "a plane pass gave up waiting for its data");
        }
    }
    if (res) {
        std::memset(res, 0, sizeof *res);
        res->steps_done = lo.done;
        res->early_stop = lo.early;
        res->n_energies = lo.n_en;
        res->energy = lo.energy;
        res->device_ms = ms;
        res->kernel_launches = c->launches;
        double nrm = 0;
        st = norm_now(c, c->polished ? GPUE_PREC_FP64 : c->prec, &nrm);
        if (st) return st;
        res->norm = nrm;
    }
    return GPUE_OK;
}

}  // extern "C"

namespace gpue {

int find_pass_kernels(int prec, int n, const PassKernel** out, int cap) {
    int k = 0;
    for (int part = 0; part < 2; ++part) {
        int cnt = 0;
        const PassKernel* t =
            prec == PREC_F32 ? (part ? pass_table_f32_b(&cnt) : pass_table_f32_a(&cnt))
                             : (part ? pass_table_f64_b(&cnt) : pass_table_f64_a(&cnt));
        for (int i = 0; i < cnt; ++i)
            if (t[i].n == n && k < cap) out[k++] = &t[i];
    }
    return k;
}

const PassKernel* find_pass_kernel(int prec, int n) {
    const PassKernel* k = nullptr;
    return find_pass_kernels(prec, n, &k, 1) ? k : nullptr;
}

}  // namespace gpue
