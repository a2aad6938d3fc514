// batch_internal.h -- launch planning shared by batches and the server.
//
// A run steps many contexts together.  Its solves are grouped by (precision,
// dimension, grid, launch shape, pass schedule); a group issues one
// k_pass_batch launch per logical pass over all its members' tiles, each CTA
// finding its solve in a prefix table.  Groups run on their own streams
// between a fork and a join; after the join one block evaluates every solve's
// energy check (k_batch_check) and clears the active flag of those that
// stopped, which freezes them: every later kernel skips their tiles.
//
// Solves whose every axis has a length the persistent multi-size kernel
// covers (batch_mega.cuh) take no group launches for their steps: all of them,
// whatever their sizes, run in one k_batch_mega launch per segment and
// precision, on the main stream while the other groups' lanes run.  Their
// energy passes follow on the main stream.  GPUE_BATCH_MEGA=0 keeps every
// solve on group launches.
#pragma once

#include "batch_mega.cuh"
#include "engine_internal.h"

namespace gpue_eng {

// Device storage for kernel argument arrays.
struct ArgSink {
    virtual ~ArgSink() = default;
    // copies `bytes` and returns their device address in *dev
    virtual gpue_status put(const void* data, size_t bytes, const void** dev,
                            std::string& err) = 0;
};

struct BGroup {
    int prec = 0;
    bool guard = false;
    bool mega = false;         // its solves run on the persistent multi-size kernel
    bool tile = false;         // 3D complex64: the three tile-stream passes per step, per solve
    std::vector<int> members;  // indices into BatchRun::ctx
};

struct BatchRun {
    int gstate = 0;
    int every = 0;        // steps between checks
    int step_base = 1;    // see k_batch_check
    double thr = 0;
    int thr_abs = 0;
    bool scale_step0 = false;     // renormalise (by scal[kScale]) before step 0 too
    std::vector<gpue_ctx*> ctx;   // the solves
    const CheckArgs* checks = nullptr;  // device, one per solve of ctx (k_batch_check)
    std::vector<int> offset;      // per solve: its step index at segment step 0
    std::vector<bool> guard;      // per solve: real-time norm guard
    std::vector<BGroup> groups;
};

using LaunchOp = std::function<void(cudaStream_t)>;

struct SegPlan {
    std::vector<std::vector<LaunchOp>> lanes;  // one list per group
    std::vector<LaunchOp> main_ops;            // the persistent launches and what follows them
    bool check = false;
    long launches = 0;
};

// Passes of steps [i0, i1) of one solve (imaginary-time steps after the
// first renormalise; step 0 too when scale_step0).
// plane: the 3D complex64 schedule of the tile-stream (or plane) passes.
std::vector<LPass> solve_passes(gpue_ctx* c, int i0, int i1, int gstate, bool guard,
                                bool scale_step0, bool plane = false);
// Whether a solve's steps run as the tile-stream passes in a batch: 3D
// complex64 with the XY and z tile kernels planned, at least
// GPUE_BATCH_TILE_MIN points (default 2^20: smaller grids do better sharing
// launches), GPUE_BATCH_TILE not 0.
bool tile_eligible(const gpue_ctx* c, int prec);
// Launch-relevant description of a pass list: equal strings can share launches.
std::string pass_signature(const gpue_ctx* c, int prec, const std::vector<LPass>& v);
// Groups r.ctx by the signature of steps [0, probe) from each solve's offset.
void group_solves(BatchRun& r, int probe);
// Plans segment steps [s0, s1) (relative to each solve's offset) plus, when
// `check`, the energy passes; argument arrays go to `sink`.
gpue_status plan_segment(const BatchRun& r, int s0, int s1, bool check, ArgSink& sink,
                         SegPlan& sp, std::string& err);
// Streams and events the launches of a segment need.
struct Lanes {
    cudaEvent_t fork = nullptr;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> joins;
    gpue_status ensure(size_t n, std::string& err);
    void destroy();
};
// Enqueues a planned segment on `main`: groups fork onto lanes, join back,
// then k_batch_check over all solves (r.checks, else `checks`) when the
// segment has a check.
void enqueue_segment(const SegPlan& sp, const BatchRun& r, cudaStream_t main, Lanes& lanes,
                     const CheckArgs* checks, int* nactive);

}  // namespace gpue_eng
