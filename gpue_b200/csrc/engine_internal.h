// engine_internal.h -- context internals shared by the engine, batch and
// server translation units (not part of the public ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gpue_b200.h"
#include "ast.h"
#include "aux_kernels.cuh"
#include "registry.h"

namespace gpue_eng {

using namespace gpue;


const double kPI = 3.141592653589793;  // GPUE's PI (include/constants.h)

struct Axis {
    int n = 1;
    double xmax = 0, dx = 1;
    std::vector<double> x, p;  // positions, momenta (generate_p_space order)
};

// Device tables for one precision.
struct Tables {
    void* buf = nullptr;
    const double2* vfac[3] = {};
    const double2* kfac[3] = {};
    const void* tw[3] = {};
    const double* pos[3] = {};
    const double* mom[3] = {};
    const double* vreal[3] = {};
    const float2* vd[3] = {};   // complex64 forms: V/2 and K factors minus 1, as float2
    const float2* kd[3] = {};
    int built_for = -1;  // gstate of vfac/kfac
};

struct LaunchCfg {
    const PassKernel* k = nullptr;
    int threads = 0, blocks = 0;
    int lines = 0;          // lines per tile (CTA)
    long ntiles = 0;
    size_t smem = 0;
    bool tuned = false;     // chosen by the autotuner
    float us = 0, default_us = 0;  // tuned and default pass times (FFT round trip)
};

// XY-plane passes of a 3D context (plane.cuh): the kernel pair and the
// persistent grid (whole clusters)
struct PlaneCfg {
    const PlaneKernel* k = nullptr;
    int blocks = 0;
};
// LPass::axis values of the two plane passes
enum { kPlaneFwd = 3, kPlaneInv = 4 };

// Work counters of a tile-stream pass (tstream.cuh): ticket (8 bytes),
// finish count (4 bytes, padded to 8), one int per z-plane; cleared once at
// allocation, then by each launch's last CTA
struct TSCounters {
    void* mem = nullptr;
    size_t bytes = 0;
    int lag = 64;  // XY pass: planes between a plane's x-tiles and its y-tiles
    // XY pass: x-tiles beyond a plane's own that its y-tiles wait for: 0, or
    // (GPUE_TEST_PLANE_WAIT, for tests only) more than ever come, so every
    // such wait runs out and the run reports GPUE_ERR_TIMEOUT
    int wait_extra = 0;
    XYCounters dev() const {
        XYCounters k;
        k.lag = lag;
        k.wait_extra = wait_extra;
        k.ticket = static_cast<unsigned long long*>(mem);
        k.finish = reinterpret_cast<unsigned*>(static_cast<char*>(mem) + 8);
        k.done_x = reinterpret_cast<int*>(static_cast<char*>(mem) + 16);
        return k;
    }
};

// The XY pass of a 3D context (tstream.cuh): the kernel pair, the x-tile and
// y-tile tensor maps of the resident field and the work counters
struct XYCfg {
    const XYKernel* k = nullptr;
    CUtensorMap tmx, tmy;
    int blocks = 0;
    TSCounters ctr;
};

// The TMA z pass of a 3D context (tstream.cuh): the kernel, the z-tile tensor
// map of the context's resident field and the work counters
struct ZCfg {
    const ZPassKernel* k = nullptr;
    CUtensorMap tm;
    int blocks = 0;
    TSCounters ctr;
};

struct GraphKey {
    int prec, gstate, parity, nsteps, scale_first, energy_last, guard, observables;
    bool operator<(const GraphKey& o) const {
        return std::memcmp(this, &o, sizeof(GraphKey)) < 0;
    }
};

struct Segment {
    cudaGraphExec_t exec = nullptr;
    long launches = 0;
};


}  // namespace gpue_eng

struct gpue_ctx {
    gpue_params p{};
    int dim = 2;
    int prec = GPUE_PREC_FP64;
    gpue_eng::Axis ax[3];
    long N = 0;
    double dV = 1;
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    void* psi = nullptr;      // resident state in the context precision
    void* psi64 = nullptr;    // FP64 shadow of an FP32 context (polishing)
    bool polished = false;    // psi64 holds the authoritative state
    void* scratch = nullptr;  // N * 16 bytes
    double* scal = nullptr;   // device scalars
    double2* partials = nullptr;
    long partials_cap = 0;
    unsigned* counters = nullptr;
    int* dflags = nullptr;       // [0] active (batched runs), [1] steps when converged,
                                 // [3] a bounded device wait gave up
    gpue_eng::Tables tab[2];            // indexed by GPUE_PREC_*
    gpue_eng::LaunchCfg lc[2][3];       // [precision][axis]
    gpue_eng::PlaneCfg plane[2];        // [precision]: XY-plane passes, if any
    gpue_eng::ZCfg zpass[2];            // [precision]: the TMA z pass, if any
    gpue_eng::XYCfg xy[2];              // [precision]: the cluster-free XY pass, if any
    bool have_wfc = false;
    bool pending_scale = false;  // scal[kScale] must multiply psi
    std::map<gpue_eng::GraphKey, gpue_eng::Segment> graphs;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    long launches = 0;         // kernels enqueued in the current evolve call
    double last_energy = 0.0;  // energy of the latest check (GPUE's "energy" key)
    // parameter-file fields (gpue_load_param_text)
    bool ext = false;          // passes use the table / expression forms
    double* vtab = nullptr;    // static V(g) and A_a(g) (FP64, N each)
    double* atab[3] = {};
    bool use_atab = false;     // gauge from the A tables instead of the rotation preset
    bool atab_nonzero[3] = {};
    gpue::AstInstr* progs = nullptr; // device copy of the time-dependent programs
    int prog_off[5] = {-1, -1, -1, -1, -1};  // V, k, Ax, Ay, Az
    int prog_len[5] = {};
    bool time_dep = false;     // some factor is evaluated per step
    // gpue_set_check_observables: observables at every energy check
    gpue_observables* obs_out = nullptr;  // caller's array, obs_cap entries
    int obs_cap = 0;
    double* obs_dev = nullptr;            // the reduction's kObsN results
    void* vtx_ws = nullptr;    // gpue_find_vortices workspace (allocated on first use)
    size_t vtx_ws_bytes = 0;
};

namespace gpue_eng {


// device scalar slots
enum {
    kScale = 0,       // imaginary-time renormalisation factor
    kEkin = 1,
    kEreal = 2,
    kNorm = 3,
    kGuard = 4,       // real-time norm-guard factor
    kTargetImag = 5,  // 1/dV: sum |psi|^2 of a unit-norm state
    kTargetReal = 6,  // sum |psi|^2 at the start of a real-time evolve
    kOne = 7,
    kEold = 8,        // batched runs: energy of the previous check
    kEcheck = 9,      // batched runs: energy of the latest check
    kNScal = 16
};
// counter slots: reductions in flight in one stream use distinct counters
enum { kCtrNorm = 0, kCtrEkin = 1, kCtrEreal = 2, kCtrMisc = 3, kNCtr = 8 };
constexpr long kAuxPartials = 4096;  // partials reserved for the aux kernels

// Records a message on the context and returns st.
gpue_status fail(gpue_ctx* c, gpue_status st, const char* fmt, ...);

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(c, e_ == cudaErrorMemoryAllocation ? GPUE_ERR_OUT_OF_MEMORY      \
                                                           : GPUE_ERR_CUDA,              \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,       \
                        __LINE__);                                                       \
    } while (0)

struct LPass {
    int axis = 0;
    std::vector<int> ops;
    int red = RED_NONE;       // RED_NONE / RED_NORM / RED_SUM
    bool red_blocks = true;   // the next pass needs the reduction result
    int red_slot = 0;         // scalar slot for the result
    int red_target = kTargetImag;
    int ctr = 0;              // counter slot
    bool store = true;
    bool to_scratch = false;   // out = scratch
    bool from_scratch = false; // in = scratch
    double gauge_dt = 0;       // for OP_GAUGE
    int scale_slot = kScale;   // OP_SCALE factor
    int kscale_slot = -1;      // extra factor folded into OP_KPHASE (norm guard)
    double time = 0;           // Dt * step, for time-dependent expressions
};

// Launches a kernel; with `pdl` it may start while the previous kernel in the
// stream is finishing (programmatic dependent launch): only for pass kernels
// that follow a pass kernel, which wait for their predecessor (pdl_wait).
template <typename... P, typename... A>
inline cudaError_t launch_kernel(void (*fn)(P...), unsigned grid, unsigned threads, size_t smem,
                                 cudaStream_t s, bool pdl, A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, fn, std::forward<A>(args)...);
}

size_t elem_size(int prec);
int kprec(int prec);
void* state_of(gpue_ctx* c, int prec);
bool axis_gauge_active(const gpue_ctx* c, int axis);
gpue_status build_tables(gpue_ctx* c, int prec, int gstate);
gpue_status plan_axis(gpue_ctx* c, int prec, int axis);
// Times every compiled plan and lines-per-CTA choice for the context's grid
// and keeps the fastest for each axis (cached per shape for the process).
gpue_status autotune_ctx(gpue_ctx* c, int prec, bool force);
gpue_status make_pass_args(gpue_ctx* c, int prec, const LPass& lp, int gstate, PassArgs& a);
// A tile-stream launch (tstream.cuh): the kernel, the context's tensor maps
// (they live as long as the context), the work counters and the grid.
struct TileLaunch {
    const void* fn = nullptr;
    const CUtensorMap* tm0 = nullptr;
    const CUtensorMap* tm1 = nullptr;
    XYCounters kc{};
    int blocks = 0, threads = 0;
    size_t smem = 0;
};
// Whether pass lp of c runs as a tile-stream kernel (the XY passes, and the
// in-place F K I z pass, where planned), and that launch.
bool tile_pass(gpue_ctx* c, int prec, const LPass& lp, const PassArgs& a, TileLaunch& t);
cudaError_t launch_tile(const TileLaunch& t, const PassArgs& a, cudaStream_t s, bool pdl);
// plane: run the in-plane axes of a 3D step as the two XY-plane passes
void step_passes(gpue_ctx* c, int i, int gstate, bool scale_first, double rexp, int guard,
                 std::vector<LPass>& out, bool plane = false);
// Plans the XY-plane passes of precision prec when the context qualifies
// (3D, nx = ny with a compiled plane kernel); leaves them off otherwise.
gpue_status plan_plane(gpue_ctx* c, int prec);
// Plans the TMA z pass of precision prec when the context qualifies (3D, nx a
// multiple of 16, nz <= 256 with a compiled kernel).
gpue_status plan_zpass(gpue_ctx* c, int prec);
// Plans the cluster-free XY pass (3D, nx = ny <= 256 with a compiled kernel);
// when planned it runs the plane passes of the step instead of the cluster
// kernels.
gpue_status plan_xy(gpue_ctx* c, int prec);
// The plane passes can run this context's steps now (no table or expression
// fields, no in-plane gauge).
bool plane_ok(const gpue_ctx* c, int prec);
void fuse(std::vector<LPass>& v);
std::vector<LPass> energy_passes(const gpue_ctx* c, bool scale_pending);
EnergyArgs energy_args(gpue_ctx* c, int prec, bool scale_pending);
gpue_status scale_state(gpue_ctx* c, int prec, int slot);
gpue_status apply_pending_scale(gpue_ctx* c, int prec);
gpue_status norm_to_slot(gpue_ctx* c, int prec, int slot);
gpue_status unpolish(gpue_ctx* c);
// device bytes a context holds (state, scratch, tables, reduction buffers),
// and the same for a fresh context of the given shape and precision
size_t ctx_device_bytes(const gpue_ctx* c);
size_t ctx_bytes_estimate(int dim, int n, int prec);

}  // namespace gpue_eng
