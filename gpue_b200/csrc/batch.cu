// batch.cu -- many independent solves stepped together (gpue_batch_*), and
// the launch planner the batch and the server share (batch_internal.h).
//
// A batch follows evolve()'s schedule for every solve at once: checks after
// steps k*every (src/evolution.cu:872-905), cut into segments that end right
// after each check step.  Segments of equal shape are captured once as a CUDA
// graph and replayed; kernel argument arrays live in device chunks owned by
// the batch, shared between graphs when equal.

#include "batch_internal.h"

using namespace gpue;
using namespace gpue_eng;

// ================================================================ planner ==

namespace gpue_eng {

std::vector<LPass> solve_passes(gpue_ctx* c, int i0, int i1, int gstate, bool guard,
                                bool scale_step0, bool plane) {
    std::vector<LPass> v;
    for (int i = i0; i < i1; ++i)
        step_passes(c, i, gstate, gstate == 0 && (i > 0 || scale_step0), 1.0, guard, v, plane);
    fuse(v);
    return v;
}

std::string pass_signature(const gpue_ctx* c, int prec, const std::vector<LPass>& v) {
    std::string s;
    auto put = [&](long x) { s += std::to_string(x) + ","; };
    put(prec);
    put(c->dim);
    for (int a = 0; a < c->dim; ++a) {
        const LaunchCfg& lc = c->lc[prec][a];
        put(c->ax[a].n);
        if (lc.k) {
            put(lc.k->ra);
            put(lc.k->rb);
            put(lc.k->rc);
            put(lc.k->p);
        }
        put(lc.threads);
        put(lc.ntiles);
        put((long)lc.smem);
    }
    for (const LPass& lp : v) {
        s += "|";
        put(lp.axis);
        for (int op : lp.ops) put(op);
        put(lp.red);
        put(lp.red_blocks);
        put(lp.red_slot);
        put(lp.red_target);
        put(lp.ctr);
        put(lp.store);
        put(lp.to_scratch);
        put(lp.from_scratch);
        put(lp.scale_slot);
        put(lp.kscale_slot);
    }
    return s;
}

// Lines per tile of a persistent-kernel tile body, and whether the solve's
// every axis has a body that tiles it.
int mega_lines(int kind) { return kMegaThreads / mega_threads_per_line(kind); }

bool mega_eligible(const gpue_ctx* c, int prec) {
    const char* env = std::getenv("GPUE_BATCH_MEGA");
    if (env && env[0] == '0') return false;
    if (c->ext || c->time_dep) return false;
    for (int a = 0; a < c->dim; ++a) {
        const int kind = mega_kind(kprec(prec), c->ax[a].n, a);
        if (kind < 0 || mega_plan_ls(kprec(prec), kind) < 0) return false;
        const int C = mega_lines(kind);
        const long nlines = c->N / c->ax[a].n;
        if (nlines % C || (a > 0 && c->ax[0].n % C)) return false;
    }
    return true;
}

bool tile_eligible(const gpue_ctx* c, int prec) {
    const char* env = std::getenv("GPUE_BATCH_TILE");
    if (env && env[0] == '0') return false;
    long min_points = 1L << 20;
    if (const char* m = std::getenv("GPUE_BATCH_TILE_MIN")) min_points = std::atol(m);
    return prec == GPUE_PREC_FP32 && c->dim == 3 && !c->time_dep && c->N >= min_points &&
           c->xy[prec].k && c->zpass[prec].k && plane_ok(c, prec);
}

void group_solves(BatchRun& r, int probe) {
    r.groups.clear();
    std::map<std::string, int> by_sig;
    for (size_t i = 0; i < r.ctx.size(); ++i) {
        gpue_ctx* c = r.ctx[i];
        const int off = r.offset[i];
        const bool tile = tile_eligible(c, c->prec);
        const std::string sig =
            std::to_string((int)r.guard[i]) + "/" + (tile ? "tile/" : "") +
            pass_signature(c, c->prec,
                           solve_passes(c, off, off + probe, r.gstate, r.guard[i], r.scale_step0,
                                        tile));
        auto it = by_sig.find(sig);
        if (it == by_sig.end()) {
            it = by_sig.emplace(sig, (int)r.groups.size()).first;
            BGroup g;
            g.prec = c->prec;
            g.guard = r.guard[i];
            g.tile = tile;
            g.mega = !tile && mega_eligible(c, c->prec);
            r.groups.push_back(g);
        }
        r.groups[it->second].members.push_back((int)i);
    }
}

namespace {

gpue_status set_batch_smem(const void* fn, size_t smem, std::string& err) {
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) {
            err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
            return GPUE_ERR_CUDA;
        }
    }
    return GPUE_OK;
}

}  // namespace

// One k_batch_mega launch for the steps [s0, s1) of every persistent-kernel
// solve of precision `prec` (after a clear of its counters), appended to ops.
gpue_status plan_mega(const BatchRun& r, int prec, int s0, int s1, ArgSink& sink,
                      std::vector<LaunchOp>& ops, long& launches, std::string& err) {
    std::vector<int> solves;
    for (const BGroup& g : r.groups)
        if (g.mega && g.prec == prec)
            for (int m : g.members) solves.push_back(m);
    if (solves.empty()) return GPUE_OK;
    const int ns = (int)solves.size();
    std::vector<std::vector<LPass>> lists(ns);
    size_t depth = 0;  // the longest pass list
    for (int k = 0; k < ns; ++k) {
        const int m = solves[k];
        lists[k] = solve_passes(r.ctx[m], r.offset[m] + s0, r.offset[m] + s1, r.gstate,
                                r.guard[m], r.scale_step0);
        depth = std::max(depth, lists[k].size());
    }
    void* fn = mega_kernel(kprec(prec));
    int per_sm = 0;
    gpue_ctx* c0 = r.ctx[solves[0]];
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kMegaThreads,
                                                      48 * 1024) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    // work items of about 32K points, fewer when the solves are too few to
    // give every resident CTA work (a converged batch's tail)
    double layer_pts = 0;  // points of one pass over all solves
    for (int k = 0; k < ns; ++k) layer_pts += (double)r.ctx[solves[k]]->N;
    const long item_pts =
        std::max(2048L, std::min(32768L, (long)(layer_pts / ((double)per_sm * c0->sms))));
    // pass instances by pass index, cut into items; argument blocks stored once
    // per content
    std::vector<MegaPass> inst;
    std::vector<int> item_pass;
    std::vector<PassArgs> args;
    std::map<std::string, int> arg_index;
    std::vector<int> last(ns, -1);
    long start = 0;
    size_t smem = 2 * (kMegaThreads / 32) * sizeof(double);
    for (size_t rd = 0; rd < depth; ++rd) {
        for (int k = 0; k < ns; ++k) {
            if (rd >= lists[k].size()) continue;
            gpue_ctx* c = r.ctx[solves[k]];
            const LPass& lp = lists[k][rd];
            PassArgs a;
            gpue_status st = make_pass_args(c, prec, lp, r.gstate, a);
            if (st) {
                err = c->err;
                return st;
            }
            const int n_ax = c->ax[lp.axis].n;
            const int kind = mega_kind(kprec(prec), n_ax, lp.axis);
            const int C = mega_lines(kind);
            a.ntiles = (c->N / n_ax) / C;
            smem = std::max(smem, (size_t)C * mega_plan_ls(kprec(prec), kind) * elem_size(prec));
            const std::string key(reinterpret_cast<const char*>(&a), sizeof a);
            auto it = arg_index.find(key);
            if (it == arg_index.end()) {
                it = arg_index.emplace(key, (int)args.size()).first;
                args.push_back(a);
            }
            MegaPass p;
            p.start = start;
            p.ntiles = (int)a.ntiles;
            p.chunk = std::max(1, (int)(item_pts / ((long)C * n_ax)));
            p.nitems = (p.ntiles + p.chunk - 1) / p.chunk;
            p.dep = last[k];
            p.kind = kind;
            p.args = it->second;
            last[k] = (int)inst.size();
            for (int i = 0; i < p.nitems; ++i) item_pass.push_back((int)inst.size());
            inst.push_back(p);
            start += p.nitems;
        }
    }
    // counters: the ticket (8 bytes) and one completion count per instance
    std::vector<int> zeros(2 + inst.size(), 0);
    const void *dinst, *ditems, *dargs, *dctr;
    gpue_status st = sink.put(inst.data(), inst.size() * sizeof(MegaPass), &dinst, err);
    if (!st) st = sink.put(item_pass.data(), item_pass.size() * sizeof(int), &ditems, err);
    if (!st) st = sink.put(args.data(), args.size() * sizeof(PassArgs), &dargs, err);
    if (!st) st = sink.put(zeros.data(), zeros.size() * sizeof(int), &dctr, err);
    if (st) return st;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) {
            err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
            return GPUE_ERR_CUDA;
        }
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kMegaThreads, smem) !=
            cudaSuccess || per_sm < 1) {
        err = "no resident launch shape for the persistent batched kernel";
        return GPUE_ERR_CUDA;
    }
    const long grid = std::min<long>((long)per_sm * c0->sms, start);
    MegaArgs ma;
    ma.passes = static_cast<const MegaPass*>(dinst);
    ma.item_pass = static_cast<const int*>(ditems);
    ma.npass = (int)inst.size();
    ma.total = start;
    ma.args = static_cast<const PassArgs*>(dargs);
    ma.ticket = reinterpret_cast<unsigned long long*>(const_cast<void*>(dctr));
    ma.done = reinterpret_cast<int*>(const_cast<void*>(dctr)) + 2;
    ma.err = c0->dflags + 3;
    const size_t ctr_bytes = zeros.size() * sizeof(int);
    void* ctr = const_cast<void*>(dctr);
    ops.push_back([=](cudaStream_t s) {
        cudaMemsetAsync(ctr, 0, ctr_bytes, s);
        void* params[] = {const_cast<MegaArgs*>(&ma)};
        cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(kMegaThreads), params, smem, s);
    });
    launches++;
    return GPUE_OK;
}

gpue_status plan_segment(const BatchRun& r, int s0, int s1, bool check, ArgSink& sink,
                         SegPlan& sp, std::string& err) {
    sp.lanes.assign(r.groups.size(), {});
    sp.main_ops.clear();
    sp.check = check;
    sp.launches = 0;
    for (int prec : {GPUE_PREC_FP64, GPUE_PREC_FP32}) {
        gpue_status st = plan_mega(r, prec, s0, s1, sink, sp.main_ops, sp.launches, err);
        if (st) return st;
    }
    for (size_t gi = 0; gi < r.groups.size(); ++gi) {
        const BGroup& g = r.groups[gi];
        // persistent-kernel groups only add their energy passes, after it
        if (g.mega && !check) continue;
        std::vector<LaunchOp>& out_ops = g.mega ? sp.main_ops : sp.lanes[gi];
        const int n = (int)g.members.size();
        gpue_ctx* c0 = r.ctx[g.members[0]];
        std::vector<std::vector<LPass>> lists(n);
        for (int k = 0; k < n; ++k) {
            const int m = g.members[k];
            gpue_ctx* c = r.ctx[m];
            if (!g.mega)
                lists[k] = solve_passes(c, r.offset[m] + s0, r.offset[m] + s1, r.gstate,
                                        r.guard[m], r.scale_step0, g.tile);
            if (check)
                for (const LPass& lp : energy_passes(c, r.gstate == 0)) lists[k].push_back(lp);
        }
        const size_t npass = lists[0].size();
        std::vector<PassArgs> args(n);
        std::vector<long> prefix(n);
        for (size_t j = 0; j < npass; ++j) {
            const int axis = lists[0][j].axis;
            for (int k = 0; k < n; ++k) {
                gpue_ctx* c = r.ctx[g.members[k]];
                if (lists[k].size() != npass || lists[k][j].axis != axis) {
                    err = "batch group schedules differ";
                    return GPUE_ERR_STATE;
                }
                gpue_status st = make_pass_args(c, g.prec, lists[k][j], r.gstate, args[k]);
                if (st) {
                    err = c->err;
                    return st;
                }
            }
            // tile-stream passes: one launch per solve (its own tensor maps and
            // counters); a converged solve's launch returns at once
            TileLaunch tl0;
            if (g.tile && tile_pass(c0, g.prec, lists[0][j], args[0], tl0)) {
                for (int k = 0; k < n; ++k) {
                    gpue_ctx* c = r.ctx[g.members[k]];
                    TileLaunch tl;
                    if (!tile_pass(c, g.prec, lists[k][j], args[k], tl)) {
                        err = "batch group tile passes differ";
                        return GPUE_ERR_STATE;
                    }
                    const PassArgs a = args[k];
                    const bool pdl = j > 0 || k > 0;  // follows a pass kernel on this lane
                    out_ops.push_back([=](cudaStream_t s) { launch_tile(tl, a, s, pdl); });
                    sp.launches++;
                }
                continue;
            }
            if (axis >= kPlaneFwd) {
                err = "batch group plane pass without a tile kernel";
                return GPUE_ERR_STATE;
            }
            const LaunchCfg& lc = c0->lc[g.prec][axis];
            for (int k = 0; k < n; ++k) prefix[k] = (long)k * lc.ntiles;
            const void *dargs, *dprefix;
            gpue_status st = sink.put(args.data(), n * sizeof(PassArgs), &dargs, err);
            if (st) return st;
            st = sink.put(prefix.data(), n * sizeof(long), &dprefix, err);
            if (st) return st;
            void (*fn)(const PassArgs*, const long*, int) =
                axis == 0 ? lc.k->row_batch : lc.k->col_batch;
            st = set_batch_smem((const void*)fn, lc.smem, err);
            if (st) return st;
            const unsigned grid = (unsigned)(n * lc.ntiles);
            const unsigned threads = (unsigned)lc.threads;
            const size_t smem = lc.smem;
            const bool pdl = j > 0;  // follows a pass kernel on this lane
            out_ops.push_back([=](cudaStream_t s) {
                launch_kernel(fn, grid, threads, smem, s, pdl,
                              static_cast<const PassArgs*>(dargs),
                              static_cast<const long*>(dprefix), n);
            });
            sp.launches++;
        }
        if (check) {
            std::vector<EnergyArgs> ea(n);
            std::vector<const int*> act(n);
            for (int k = 0; k < n; ++k) {
                gpue_ctx* c = r.ctx[g.members[k]];
                ea[k] = energy_args(c, g.prec, r.gstate == 0);
                act[k] = c->dflags;
            }
            const void *dea, *dact;
            gpue_status st = sink.put(ea.data(), n * sizeof(EnergyArgs), &dea, err);
            if (st) return st;
            st = sink.put(act.data(), n * sizeof(const int*), &dact, err);
            if (st) return st;
            long per = c0->N / (256 * 8);
            per = std::max(1L, std::min(per, kAuxPartials));
            const unsigned grid = (unsigned)(n * per);
            const int iper = (int)per;
            const bool f32 = g.prec == GPUE_PREC_FP32;
            out_ops.push_back([=](cudaStream_t s) {
                const EnergyArgs* e = static_cast<const EnergyArgs*>(dea);
                const int* const* a = static_cast<const int* const*>(dact);
                if (f32) k_energy_real_batch<float><<<grid, 256, 0, s>>>(e, a, iper);
                else k_energy_real_batch<double><<<grid, 256, 0, s>>>(e, a, iper);
            });
            sp.launches++;
        }
    }
    if (check) sp.launches++;  // k_batch_check
    return GPUE_OK;
}

gpue_status Lanes::ensure(size_t n, std::string& err) {
    auto ck = [&](cudaError_t e) {
        if (e == cudaSuccess) return false;
        err = std::string("lane setup: ") + cudaGetErrorString(e);
        return true;
    };
    if (!fork && ck(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming))) return GPUE_ERR_CUDA;
    while (streams.size() < n) {
        cudaStream_t s;
        cudaEvent_t e;
        if (ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking))) return GPUE_ERR_CUDA;
        if (ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming))) {
            cudaStreamDestroy(s);
            return GPUE_ERR_CUDA;
        }
        streams.push_back(s);
        joins.push_back(e);
    }
    return GPUE_OK;
}

void Lanes::destroy() {
    for (auto s : streams) cudaStreamDestroy(s);
    for (auto e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    streams.clear();
    joins.clear();
    fork = nullptr;
}

void enqueue_segment(const SegPlan& sp, const BatchRun& r, cudaStream_t main, Lanes& lanes,
                     const CheckArgs* checks, int* nactive) {
    cudaEventRecord(lanes.fork, main);
    for (size_t gi = 0; gi < sp.lanes.size(); ++gi) {
        if (sp.lanes[gi].empty()) continue;
        cudaStream_t s = lanes.streams[gi];
        cudaStreamWaitEvent(s, lanes.fork, 0);
        for (const LaunchOp& op : sp.lanes[gi]) op(s);
        cudaEventRecord(lanes.joins[gi], s);
    }
    // the persistent launches run on the main stream while the lanes run
    for (const LaunchOp& op : sp.main_ops) op(main);
    for (size_t gi = 0; gi < sp.lanes.size(); ++gi)
        if (!sp.lanes[gi].empty()) cudaStreamWaitEvent(main, lanes.joins[gi], 0);
    if (sp.check)
        k_batch_check<<<1, 256, 0, main>>>(r.checks ? r.checks : checks, (int)r.ctx.size(),
                                            r.every, r.step_base,
                                            r.thr, r.thr_abs, r.gstate == 0 ? 1 : 0, nactive);
}

}  // namespace gpue_eng

// ================================================================ batches ==

namespace {

// Argument arrays for captured graphs: equal arrays share storage, which
// lives as long as the batch.
struct ChunkSink : ArgSink {
    std::vector<std::pair<char*, size_t>> chunks;
    size_t used = 0;
    std::map<std::string, const void*> stored;

    gpue_status put(const void* data, size_t bytes, const void** out, std::string& err) override {
        std::string key(static_cast<const char*>(data), bytes);
        auto it = stored.find(key);
        if (it != stored.end()) {
            *out = it->second;
            return GPUE_OK;
        }
        const size_t need = (bytes + 255) & ~size_t(255);
        if (chunks.empty() || used + need > chunks.back().second) {
            const size_t cap = std::max<size_t>(size_t(4) << 20, need);
            char* p = nullptr;
            cudaError_t e = cudaMalloc(&p, cap);
            if (e != cudaSuccess) {
                err = std::string("argument storage: ") + cudaGetErrorString(e);
                return e == cudaErrorMemoryAllocation ? GPUE_ERR_OUT_OF_MEMORY : GPUE_ERR_CUDA;
            }
            chunks.emplace_back(p, cap);
            used = 0;
        }
        char* dst = chunks.back().first + used;
        cudaError_t e = cudaMemcpy(dst, data, bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            err = std::string("argument upload: ") + cudaGetErrorString(e);
            return GPUE_ERR_CUDA;
        }
        used += need;
        stored.emplace(std::move(key), dst);
        *out = dst;
        return GPUE_OK;
    }

    ~ChunkSink() override {
        for (auto& ch : chunks) cudaFree(ch.first);
    }
};

}  // namespace

struct gpue_batch {
    std::vector<gpue_ctx*> ctx;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t polled[2] = {nullptr, nullptr};
    Lanes lanes;
    ChunkSink args;
    CheckArgs* checks = nullptr;  // device, one per solve
    BatchOut* outs = nullptr;     // device
    BatchOut* h_outs = nullptr;   // pinned
    int* nactive = nullptr;       // device
    int* h_nactive = nullptr;     // pinned, two slots (alternating polls)
    std::map<std::string, Segment> graphs;
    std::string err;
};

namespace {

gpue_status bfail(gpue_batch* b, gpue_status st, const char* fmt, ...) {
    if (b) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        b->err = buf;
    }
    return st;
}

#define BCK(call)                                                                        \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return bfail(b, e_ == cudaErrorMemoryAllocation ? GPUE_ERR_OUT_OF_MEMORY     \
                                                            : GPUE_ERR_CUDA,             \
                         "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,      \
                         __LINE__);                                                      \
    } while (0)

// a context error surfaces as the batch error
#define BCTX(c, call)         \
    do {                      \
        gpue_status s_ = (call); \
        if (s_) {             \
            b->err = (c)->err; \
            return s_;        \
        }                     \
    } while (0)

// Captures a list of planned segments into one graph.
gpue_status capture_segments(gpue_batch* b, const BatchRun& r, const std::vector<SegPlan>& segs,
                             Segment& out) {
    gpue_status st = b->lanes.ensure(r.groups.size(), b->err);
    if (st) return st;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    long launches = 0;
    for (const SegPlan& sp : segs) {
        enqueue_segment(sp, r, b->stream, b->lanes, b->checks, b->nactive);
        launches += sp.launches;
    }
    cudaGraph_t g = nullptr;
    BCK(cudaStreamEndCapture(b->stream, &g));
    BCK(cudaGetLastError());
    cudaError_t ce = cudaGraphInstantiate(&out.exec, g, 0);
    cudaGraphDestroy(g);
    BCK(ce);
    out.launches = launches;
    return GPUE_OK;
}

struct SegSpec {
    int i0, i1;
    bool check;
};

// evolve()'s schedule cut into segments: a check after step k*every (k >= 0)
// ends a segment; unchecked stretches are cut into at most `chunk` steps.
std::vector<SegSpec> batch_schedule(int nsteps, int every, int chunk) {
    std::vector<SegSpec> v;
    int i = 0;
    while (i < nsteps) {
        int end = std::min(nsteps, i + chunk);
        bool check = false;
        if (every > 0) {
            const int nc = ((i + every - 1) / every) * every;  // next check step >= i
            if (nc < nsteps && nc + 1 <= end) {
                end = nc + 1;
                check = true;
            }
        }
        v.push_back({i, end, check});
        i = end;
    }
    return v;
}

void destroy_batch_graphs(gpue_batch* b) {
    for (auto& kv : b->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    b->graphs.clear();
}

}  // namespace

extern "C" {

const char* gpue_batch_last_error(const gpue_batch* b) { return b ? b->err.c_str() : ""; }

gpue_status gpue_batch_create(gpue_ctx* const* ctxs, int32_t n, gpue_batch** out) {
    if (!ctxs || n < 1 || !out) return GPUE_ERR_INVALID_ARG;
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!ctxs[i] || ctxs[i]->device != ctxs[0]->device) return GPUE_ERR_INVALID_ARG;
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i]) return GPUE_ERR_INVALID_ARG;
    }
    std::unique_ptr<gpue_batch> bp(new gpue_batch);
    gpue_batch* b = bp.get();
    b->ctx.assign(ctxs, ctxs + n);
    b->device = ctxs[0]->device;
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BCK(cudaEventCreate(&b->ev0));
    BCK(cudaEventCreate(&b->ev1));
    for (auto& e : b->polled) BCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    BCK(cudaMalloc(&b->checks, n * sizeof(CheckArgs)));
    BCK(cudaMalloc(&b->outs, n * sizeof(BatchOut)));
    BCK(cudaMallocHost(&b->h_outs, n * sizeof(BatchOut)));
    BCK(cudaMalloc(&b->nactive, sizeof(int)));
    BCK(cudaMallocHost(&b->h_nactive, 2 * sizeof(int)));
    std::vector<CheckArgs> h(n);
    for (int i = 0; i < n; ++i) {
        gpue_ctx* c = ctxs[i];
        h[i].scal = c->scal;
        h[i].flags = c->dflags;
        h[i].inv_n = 1.0 / (double)c->N;
        h[i].dV = c->dV;
        h[i].slot_ekin = kEkin;
        h[i].slot_ereal = kEreal;
        h[i].slot_eold = kEold;
        h[i].slot_e = kEcheck;
    }
    BCK(cudaMemcpy(b->checks, h.data(), n * sizeof(CheckArgs), cudaMemcpyHostToDevice));
    *out = bp.release();
    return GPUE_OK;
}

gpue_status gpue_batch_destroy(gpue_batch* b) {
    if (!b) return GPUE_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    destroy_batch_graphs(b);
    b->lanes.destroy();
    cudaFree(b->checks);
    cudaFree(b->outs);
    cudaFreeHost(b->h_outs);
    cudaFree(b->nactive);
    cudaFreeHost(b->h_nactive);
    for (auto e : {b->ev0, b->ev1, b->polled[0], b->polled[1]})
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return GPUE_OK;
}

gpue_status gpue_batch_evolve(gpue_batch* b, int32_t gstate, const gpue_batch_opts* opts,
                              gpue_batch_result* results, gpue_batch_stats* stats) {
    if (!b || (gstate != 0 && gstate != 1)) return GPUE_ERR_INVALID_ARG;
    gpue_batch_opts o;
    std::memset(&o, 0, sizeof o);
    o.norm_guard = -1;
    o.max_steps = 1;
    if (opts) o = *opts;
    if (o.max_steps < 1 || o.energy_calc_steps < 0 || o.segments_per_launch < 0)
        return bfail(b, GPUE_ERR_INVALID_ARG, "invalid batch options");
    BCK(cudaSetDevice(b->device));
    const int n = (int)b->ctx.size();
    BatchRun r;
    r.gstate = gstate;
    r.every = o.energy_calc_steps;
    r.step_base = 1;
    r.thr = o.energy_calc_threshold;
    r.thr_abs = o.threshold_abs ? 1 : 0;
    r.scale_step0 = false;
    r.ctx = b->ctx;
    r.offset.assign(n, 0);
    r.guard.assign(n, false);
    double pts = 0;
    const int fresh[4] = {1, 0, 0, 0};
    for (int i = 0; i < n; ++i) {
        gpue_ctx* c = b->ctx[i];
        if (!c->have_wfc) return bfail(b, GPUE_ERR_STATE, "solve %d has no wavefunction", i);
        if (c->ext)
            return bfail(b, GPUE_ERR_UNSUPPORTED,
                         "solve %d: parameter-file fields are not batched", i);
        if (c->p.ramp && gstate == 0 && c->p.corotating &&
            (axis_gauge_active(c, 0) || axis_gauge_active(c, 1) || axis_gauge_active(c, 2)))
            return bfail(b, GPUE_ERR_UNSUPPORTED, "solve %d: the ramp is not batched", i);
        const bool guard = gstate == 1 && (o.norm_guard == 1 ||
                                           (o.norm_guard < 0 && c->prec == GPUE_PREC_FP32));
        r.guard[i] = guard;
        BCTX(c, unpolish(c));
        BCTX(c, build_tables(c, c->prec, gstate));
        if (o.autotune) BCTX(c, autotune_ctx(c, c->prec, false));
        BCTX(c, apply_pending_scale(c, c->prec));
        if (guard) {
            BCTX(c, norm_to_slot(c, c->prec, kTargetReal));
            BCK(cudaMemcpyAsync(c->scal + kGuard, c->scal + kOne, sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
        }
        BCK(cudaMemcpyAsync(c->dflags, fresh, sizeof fresh, cudaMemcpyHostToDevice, c->stream));
        BCK(cudaStreamSynchronize(c->stream));
        pts += (double)c->N;
    }
    r.checks = b->checks;
    const std::vector<bool> guard_all = r.guard;
    group_solves(r, 3);
    // graphs depend on the grouping, the members and the check parameters
    std::vector<int> ids(n);  // batch index of each solve of r
    for (int i = 0; i < n; ++i) ids[i] = i;
    auto make_key = [&](const BatchRun& run, const std::vector<int>& id) {
        std::string k = std::to_string(gstate) + ":" + std::to_string(run.every) + ":" +
                        std::to_string(run.thr_abs) + ":";
        char tb[32];
        std::snprintf(tb, sizeof tb, "%a:", run.thr);
        k += tb;
        for (const BGroup& g : run.groups) {
            k += "{" + std::to_string(g.guard) + "/" +
                 pass_signature(run.ctx[g.members[0]], g.prec,
                                solve_passes(run.ctx[g.members[0]], 0, 3, gstate, g.guard,
                                             false, g.tile)) + "}";
            for (int m : g.members) k += std::to_string(id[m]) + ",";
        }
        return k;
    };
    std::string gkey = make_key(r, ids);
    const int every = r.every;
    const std::vector<SegSpec> sched =
        batch_schedule(o.max_steps, every, every > 0 ? std::min(every + 1, 256) : 128);
    int per_launch = o.segments_per_launch;
    if (per_launch == 0) {
        // about 2e9 point-steps per graph launch, at most 16 segments
        const double seg_work = pts * (every > 0 ? every : 128);
        per_launch = (int)std::min(16.0, std::max(1.0, std::ceil(2e9 / seg_work)));
    }
    long launches = 0, glaunches = 0;
    int steps_run = 0, polls = 0;
    bool all_done = false;
    BCK(cudaEventRecord(b->ev0, b->stream));
    size_t s = 0;
    while (s < sched.size() && !all_done) {
        // consecutive segments of equal shape share one graph launch
        size_t e = s + 1;
        while (e < sched.size() && (int)(e - s) < per_launch && sched[s].i0 > 0 &&
               sched[e].i1 - sched[e].i0 == sched[s].i1 - sched[s].i0 &&
               sched[e].check == sched[s].check)
            ++e;
        std::string key = gkey + "#" + std::to_string(sched[s].i0 == 0) + "," +
                          std::to_string(sched[s].i0 % 2);
        bool has_check = false;
        for (size_t k = s; k < e; ++k) {
            key += ";" + std::to_string(sched[k].i1 - sched[k].i0) + (sched[k].check ? "c" : "");
            has_check |= sched[k].check;
        }
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            std::vector<SegPlan> plans(e - s);
            for (size_t k = s; k < e; ++k) {
                gpue_status st = plan_segment(r, sched[k].i0, sched[k].i1, sched[k].check,
                                              b->args, plans[k - s], b->err);
                if (st) return st;
            }
            Segment seg;
            gpue_status st = capture_segments(b, r, plans, seg);
            if (st) return st;
            it = b->graphs.emplace(key, seg).first;
        }
        BCK(cudaGraphLaunch(it->second.exec, b->stream));
        glaunches++;
        launches += it->second.launches;
        steps_run = sched[e - 1].i1;
        if (has_check && gstate == 0) {
            // read the previous launch's count of running solves while this one runs
            const int slot = polls % 2;
            BCK(cudaMemcpyAsync(b->h_nactive + slot, b->nactive, sizeof(int),
                                cudaMemcpyDeviceToHost, b->stream));
            BCK(cudaEventRecord(b->polled[slot], b->stream));
            int running = -1;
            if (polls > 0) {
                BCK(cudaEventSynchronize(b->polled[1 - slot]));
                running = b->h_nactive[1 - slot];
                if (running == 0) all_done = true;
            }
            polls++;
            // once half the planned solves have converged, plan the rest alone:
            // the frozen ones' work items and the coarse items of a full batch
            // would otherwise dominate the tail
            if (running > 0 && 2 * running <= (int)r.ctx.size() && e < sched.size()) {
                BCK(cudaStreamSynchronize(b->stream));
                k_batch_gather<<<(n + 127) / 128, 128, 0, b->stream>>>(b->checks, n, b->outs);
                BCK(cudaGetLastError());
                BCK(cudaMemcpyAsync(b->h_outs, b->outs, n * sizeof(BatchOut),
                                    cudaMemcpyDeviceToHost, b->stream));
                BCK(cudaStreamSynchronize(b->stream));
                BatchRun r2 = r;
                r2.ctx.clear();
                r2.offset.clear();
                r2.guard.clear();
                std::vector<int> ids2;
                std::vector<CheckArgs> ca;
                for (int i = 0; i < n; ++i) {
                    if (!b->h_outs[i].active) continue;
                    gpue_ctx* c = b->ctx[i];
                    r2.ctx.push_back(c);
                    r2.offset.push_back(0);
                    r2.guard.push_back(guard_all[i]);
                    ids2.push_back(i);
                    CheckArgs x;
                    x.scal = c->scal;
                    x.flags = c->dflags;
                    x.inv_n = 1.0 / (double)c->N;
                    x.dV = c->dV;
                    x.slot_ekin = kEkin;
                    x.slot_ereal = kEreal;
                    x.slot_eold = kEold;
                    x.slot_e = kEcheck;
                    ca.push_back(x);
                }
                if (!r2.ctx.empty()) {
                    const void* dca = nullptr;
                    gpue_status st =
                        b->args.put(ca.data(), ca.size() * sizeof(CheckArgs), &dca, b->err);
                    if (st) return st;
                    r2.checks = static_cast<const CheckArgs*>(dca);
                    group_solves(r2, 3);
                    r = r2;
                    ids = ids2;
                    gkey = make_key(r, ids);
                    polls = 0;
                }
            }
        }
        s = e;
    }
    BCK(cudaEventRecord(b->ev1, b->stream));
    k_batch_gather<<<(n + 127) / 128, 128, 0, b->stream>>>(b->checks, n, b->outs);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(b->h_outs, b->outs, n * sizeof(BatchOut), cudaMemcpyDeviceToHost,
                        b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    float ms = 0.f;
    BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    double point_steps = 0;
    for (int i = 0; i < n; ++i) {
        gpue_ctx* c = b->ctx[i];
        const BatchOut& bo = b->h_outs[i];
        const bool stopped = bo.active == 0;
        const int steps = stopped ? bo.steps : steps_run;
        point_steps += (double)c->N * steps;
        if (results) {
            results[i].steps_done = steps;
            results[i].early_stop = stopped ? 1 : 0;
            results[i].energy = bo.checks > 0 ? bo.energy : NAN;
        }
        if (bo.checks > 0) c->last_energy = bo.energy;
        if (gstate == 0) c->pending_scale = true;
        BCTX(c, apply_pending_scale(c, c->prec));
        if (guard_all[i]) BCTX(c, scale_state(c, c->prec, kGuard));
    }
    for (int i = 0; i < n; ++i) BCK(cudaStreamSynchronize(b->ctx[i]->stream));
    if (stats) {
        stats->device_ms = ms;
        stats->kernel_launches = launches;
        stats->graph_launches = glaunches;
        stats->point_steps = point_steps;
    }
    return GPUE_OK;
}

}  // extern "C"
