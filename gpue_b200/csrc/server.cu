// server.cu -- the request loop behind gpue_server_* (continuous batching).
//
// A worker thread owns the device.  Each loop it admits queued requests in
// arrival order while the HBM budget and slot limit allow (a request that
// does not fit waits at the head of the queue), then runs one tick: every
// resident solve advances check_steps steps and gets an energy check.  The
// imaginary- and real-time solves form two runs on their own streams, so
// their launches overlap on the device; within a run, solves of one shape
// share launches (batch_internal.h).  Solves that met the threshold or
// reached max_steps leave after the tick: their state is written to the
// caller's buffer, their context freed and their result queued for polling.
//
// The solves that leave at a tick return their results while the next tick
// runs (their copies use their own streams), and their contexts are freed at
// the following idle point, so the device does not wait for the copy-outs.
//
// Deadlines and cancellation are host-side: a request whose deadline has
// passed, or whose tag was cancelled, leaves the queue at once, or leaves the
// resident set after the tick in flight with its state at that tick; nothing
// waits on the device for it.
//
// A solve's step index advances by check_steps per tick from 0, so every
// solve sees evolve()'s step numbering (gauge order i % 2, renormalisation
// after each imaginary-time step) whatever tick it was admitted in, and its
// kernels reduce over its own tiles only: the arithmetic of a solve is the
// same alone and in any mix.

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <set>
#include <thread>

#include "batch_internal.h"

using namespace gpue;
using namespace gpue_eng;

namespace {

// Argument arrays of one tick, packed into pinned host memory and copied to
// the device in one transfer before the tick's launches.  Equal arrays are
// stored once.  The device buffer only changes size between ticks: a tick
// whose arrays do not fit is planned once more after the buffer has grown.
struct TickSink : ArgSink {
    char* host = nullptr;
    char* dev = nullptr;
    size_t cap = 0, used = 0;
    bool overflow = false;
    std::map<std::string, const void*> seen;

    void begin() {
        used = 0;
        overflow = false;
        seen.clear();
    }
    gpue_status put(const void* data, size_t bytes, const void** out, std::string&) override {
        std::string key(static_cast<const char*>(data), bytes);
        auto it = seen.find(key);
        if (it != seen.end()) {
            *out = it->second;
            return GPUE_OK;
        }
        const size_t need = (bytes + 255) & ~size_t(255);
        if (used + need > cap) {
            used += need;  // counts what the tick needs; the plan is discarded
            overflow = true;
            *out = nullptr;
            return GPUE_OK;
        }
        std::memcpy(host + used, data, bytes);
        *out = dev + used;
        used += need;
        seen.emplace(std::move(key), *out);
        return GPUE_OK;
    }
    gpue_status grow(size_t want, std::string& err) {
        size_t c = cap ? cap : (size_t(1) << 20);
        while (c < want) c *= 2;
        if (dev) cudaFree(dev);
        if (host) cudaFreeHost(host);
        dev = nullptr;
        host = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&dev, c);
        if (e == cudaSuccess) e = cudaMallocHost(&host, c);
        if (e != cudaSuccess) {
            err = std::string("tick arena: ") + cudaGetErrorString(e);
            return GPUE_ERR_OUT_OF_MEMORY;
        }
        cap = c;
        return GPUE_OK;
    }
    void release() {
        if (dev) cudaFree(dev);
        if (host) cudaFreeHost(host);
        dev = host = nullptr;
        cap = used = 0;
    }
};

// Streams and buffers of one run (imaginary or real time).
struct Run {
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Lanes lanes;
    TickSink sink;
    BatchOut* outs = nullptr;    // device
    BatchOut* h_outs = nullptr;  // pinned
    int* nactive = nullptr;
    size_t out_cap = 0;
    // this tick
    std::vector<int> members;  // indices into the active list
    bool issued = false;
    // The last tick captured as a graph, replayed while the run's solves
    // (and the parity of their step counts) stay the same: a tick's kernel
    // arguments then do not change, so neither planning nor upload is needed.
    cudaGraphExec_t exec = nullptr;
    std::vector<std::pair<uint64_t, int>> exec_key;  // (solve serial, step parity)
    long exec_launches = 0;
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        exec_key.clear();
        exec_launches = 0;
    }
};

struct Solve {
    uint64_t serial = 0;  // unique per admitted request (context addresses get reused)
    gpue_ctx* c = nullptr;
    gpue_request req{};
    double t_submit = 0, t_admit = 0;
    int steps = 0;
    size_t bytes = 0;
    bool guard = false;
};

struct Pending {
    gpue_request req;
    double t_submit;
};

// A solve that left the resident set at a tick: its result is written out
// while the next tick runs.
struct Leaving {
    Solve s;
    BatchOut bo;
    bool stopped;
    gpue_status why;
};

}  // namespace

struct gpue_server {
    gpue_server_opts o{};
    std::chrono::steady_clock::time_point t0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> queue;             // guarded by mu
    std::deque<gpue_server_result> done;   // guarded by mu
    std::set<int64_t> cancel;              // guarded by mu: tags of resident solves to drop
    std::multiset<int64_t> resident_tags;  // guarded by mu: admitted (or being admitted)
    gpue_server_stats st{};                // guarded by mu
    bool stop = false;                     // guarded by mu
    bool broken = false;                   // guarded by mu
    std::string err;                       // guarded by mu
    std::vector<Solve> active;             // worker only
    std::vector<Leaving> leaving;          // worker only: left at the last tick
    std::vector<Solve> zombies;            // worker only: results out, contexts to free
    Run run[2];                            // worker only
    uint64_t next_serial = 1;              // worker only
};

namespace {

double now_s(const gpue_server* S) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - S->t0).count();
}

void push_result(gpue_server* S, const gpue_server_result& r) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->done.push_back(r);
    if (r.status == GPUE_OK) S->st.completed++;
    else S->st.failed++;
    S->cv_done.notify_all();
}

gpue_server_result make_result(const gpue_request& q, gpue_status status, double t_submit,
                               double t_admit, double t_done) {
    gpue_server_result r;
    std::memset(&r, 0, sizeof r);
    r.tag = q.tag;
    r.status = status;
    r.energy = NAN;
    r.t_submit = t_submit;
    r.t_admit = t_admit;
    r.t_done = t_done;
    return r;
}

bool expired(const gpue_request& q, double t_submit, double now) {
    return q.deadline_s > 0 && now - t_submit > q.deadline_s;
}

// Drops queued requests whose deadline has passed (worker, before admission).
void drop_expired(gpue_server* S) {
    std::lock_guard<std::mutex> lk(S->mu);
    const double now = now_s(S);
    for (auto it = S->queue.begin(); it != S->queue.end();) {
        if (expired(it->req, it->t_submit, now)) {
            S->done.push_back(make_result(it->req, GPUE_ERR_TIMEOUT, it->t_submit, now, now));
            S->st.failed++;
            S->st.timed_out++;
            it = S->queue.erase(it);
        } else {
            ++it;
        }
    }
    S->cv_done.notify_all();
}

// Context of an admitted request, ready for its first tick.  With tune
// false (admission while a tick runs) no plans are timed: contention would
// skew them; shapes tuned before still get their cached choices.
gpue_status start_solve(gpue_server* S, const Pending& p, Solve& s, bool tune) {
    gpue_params prm = p.req.params;
    prm.precision = S->o.precision;
    prm.device = S->o.device;
    gpue_ctx* c = nullptr;
    gpue_status st = gpue_ctx_create(&prm, &c);
    if (st) return st;
    s.c = c;
    s.req = p.req;
    s.t_submit = p.t_submit;
    s.t_admit = now_s(S);
    s.steps = 0;
    s.guard = p.req.gstate == 1 && c->prec == GPUE_PREC_FP32;
    st = gpue_set_wfc(c, p.req.psi0, GPUE_MEM_HOST, GPUE_C128);
    if (!st) st = build_tables(c, c->prec, p.req.gstate);
    if (!st && S->o.autotune && tune) st = autotune_ctx(c, c->prec, false);
    if (!st && s.guard) {
        st = norm_to_slot(c, c->prec, kTargetReal);
        if (!st && cudaMemcpyAsync(c->scal + kGuard, c->scal + kOne, sizeof(double),
                                   cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
            st = GPUE_ERR_CUDA;
    }
    const int fresh[4] = {1, 0, 0, 0};
    if (!st && cudaMemcpyAsync(c->dflags, fresh, sizeof fresh, cudaMemcpyHostToDevice,
                               c->stream) != cudaSuccess)
        st = GPUE_ERR_CUDA;
    if (!st && cudaStreamSynchronize(c->stream) != cudaSuccess) st = GPUE_ERR_CUDA;
    s.bytes = ctx_device_bytes(c);
    return st;
}

void admit(gpue_server* S, bool tune) {
    for (;;) {
        Pending p;
        size_t est = 0;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (S->queue.empty() || S->stop) return;
            if (S->o.max_active > 0 && (int)S->active.size() >= S->o.max_active) return;
            const gpue_params& q = S->queue.front().req.params;
            est = ctx_bytes_estimate(q.dimnum, q.xDim, S->o.precision);
            const bool fits = S->st.bytes_resident + (int64_t)est <= S->st.bytes_budget;
            if (!fits && !(S->active.empty() && (int64_t)est > S->st.bytes_budget)) return;
            p = S->queue.front();
            S->queue.pop_front();
            if (fits) S->resident_tags.insert(p.req.tag);
            if (!fits) {
                // larger than the whole budget: it can never be admitted
                S->done.push_back(make_result(p.req, GPUE_ERR_OUT_OF_MEMORY, p.t_submit,
                                              now_s(S), now_s(S)));
                S->st.failed++;
                S->cv_done.notify_all();
                continue;
            }
            S->st.bytes_resident += (int64_t)est;  // reserved until the context exists
        }
        Solve s;
        gpue_status st = start_solve(S, p, s, tune);
        std::lock_guard<std::mutex> lk(S->mu);
        S->st.bytes_resident -= (int64_t)est;
        if (st) {
            auto it = S->resident_tags.find(p.req.tag);
            if (it != S->resident_tags.end()) S->resident_tags.erase(it);
            if (s.c) gpue_ctx_destroy(s.c);
            S->done.push_back(make_result(p.req, st, p.t_submit, s.t_admit, now_s(S)));
            S->st.failed++;
            S->cv_done.notify_all();
            continue;
        }
        S->st.bytes_resident += (int64_t)s.bytes;
        if (S->st.bytes_resident > S->st.bytes_peak) S->st.bytes_peak = S->st.bytes_resident;
        S->st.admitted++;
        if (!tune) S->st.admitted_in_tick++;
        S->st.active++;
        s.serial = S->next_serial++;
        S->active.push_back(s);
    }
}

// Plans and enqueues one run's tick; returns the kernels it launched.
gpue_status issue_run(gpue_server* S, int gstate, Run& R, long& launches, std::string& err) {
    R.issued = false;
    if (R.members.empty()) return GPUE_OK;
    const int n = (int)R.members.size();
    std::vector<std::pair<uint64_t, int>> key;
    key.reserve(n);
    for (int m : R.members) key.emplace_back(S->active[m].serial, S->active[m].steps % 2);
    if (R.exec && key == R.exec_key) {
        cudaEventRecord(R.e0, R.stream);
        cudaError_t e = cudaGraphLaunch(R.exec, R.stream);
        cudaEventRecord(R.e1, R.stream);
        if (e != cudaSuccess) {
            err = std::string("tick replay: ") + cudaGetErrorString(e);
            return GPUE_ERR_CUDA;
        }
        launches += R.exec_launches;
        R.issued = true;
        return GPUE_OK;
    }
    R.drop_graph();
    BatchRun r;
    r.gstate = gstate;
    r.every = S->o.check_steps;
    r.step_base = S->o.check_steps;
    r.thr = S->o.threshold;
    r.thr_abs = S->o.threshold_abs ? 1 : 0;
    r.scale_step0 = true;  // a fresh context holds scal[kScale] = 1
    for (int m : R.members) {
        r.ctx.push_back(S->active[m].c);
        r.offset.push_back(S->active[m].steps);
        r.guard.push_back(S->active[m].guard);
    }
    group_solves(r, r.every);
    SegPlan plan;
    const void* checks = nullptr;
    for (int attempt = 0;; ++attempt) {
        R.sink.begin();
        gpue_status st = plan_segment(r, 0, r.every, true, R.sink, plan, err);
        if (st == GPUE_OK) {
            std::vector<CheckArgs> ca(n);
            for (int k = 0; k < n; ++k) {
                gpue_ctx* c = r.ctx[k];
                ca[k].scal = c->scal;
                ca[k].flags = c->dflags;
                ca[k].inv_n = 1.0 / (double)c->N;
                ca[k].dV = c->dV;
                ca[k].slot_ekin = kEkin;
                ca[k].slot_ereal = kEreal;
                ca[k].slot_eold = kEold;
                ca[k].slot_e = kEcheck;
            }
            st = R.sink.put(ca.data(), n * sizeof(CheckArgs), &checks, err);
        }
        if (st) return st;
        if (!R.sink.overflow) break;
        if (attempt > 0) {
            err = "tick arena overflow";
            return GPUE_ERR_STATE;
        }
        st = R.sink.grow(R.sink.used, err);
        if (st) return st;
    }
    if ((size_t)n > R.out_cap) {
        if (R.outs) cudaFree(R.outs);
        if (R.h_outs) cudaFreeHost(R.h_outs);
        R.outs = nullptr;
        R.h_outs = nullptr;
        R.out_cap = 0;
        const size_t cap = std::max<size_t>(64, 2 * (size_t)n);
        if (cudaMalloc(&R.outs, cap * sizeof(BatchOut)) != cudaSuccess ||
            cudaMallocHost(&R.h_outs, cap * sizeof(BatchOut)) != cudaSuccess) {
            err = "tick result buffers";
            return GPUE_ERR_OUT_OF_MEMORY;
        }
        R.out_cap = cap;
    }
    gpue_status st = R.lanes.ensure(r.groups.size(), err);
    if (st) return st;
    if (cudaMemcpyAsync(R.sink.dev, R.sink.host, R.sink.used, cudaMemcpyHostToDevice,
                        R.stream) != cudaSuccess) {
        err = "tick argument upload";
        return GPUE_ERR_CUDA;
    }
    // capture the tick (launches, gather, result copy) and launch the graph
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(R.stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_segment(plan, r, R.stream, R.lanes, static_cast<const CheckArgs*>(checks),
                        R.nactive);
        k_batch_gather<<<(n + 127) / 128, 128, 0, R.stream>>>(
            static_cast<const CheckArgs*>(checks), n, R.outs);
        cudaMemcpyAsync(R.h_outs, R.outs, n * sizeof(BatchOut), cudaMemcpyDeviceToHost,
                        R.stream);
        const cudaError_t le = cudaGetLastError();
        e = cudaStreamEndCapture(R.stream, &g);
        if (e == cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&R.exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        R.exec = nullptr;
        err = std::string("tick capture: ") + cudaGetErrorString(e);
        return GPUE_ERR_CUDA;
    }
    R.exec_key = std::move(key);
    R.exec_launches = plan.launches + 1;
    cudaEventRecord(R.e0, R.stream);
    e = cudaGraphLaunch(R.exec, R.stream);
    cudaEventRecord(R.e1, R.stream);
    if (e != cudaSuccess) {
        err = std::string("tick launch: ") + cudaGetErrorString(e);
        return GPUE_ERR_CUDA;
    }
    launches += R.exec_launches;
    R.issued = true;
    return GPUE_OK;
}

// A solve's result: final scaling, copy-out, result (to push).  `why` is
// GPUE_OK for a solve that ran to its end, or the timeout / cancellation
// status of one that leaves early (its state still goes to psi_out).  Its
// context stays allocated (and counted against the budget) until release().
gpue_server_result finish(gpue_server* S, Solve& s, const BatchOut& bo, bool stopped,
                          gpue_status why = GPUE_OK) {
    gpue_ctx* c = s.c;
    gpue_status st = GPUE_OK;
    if (s.req.gstate == 0) c->pending_scale = true;
    st = apply_pending_scale(c, c->prec);
    if (!st && s.guard) st = scale_state(c, c->prec, kGuard);
    if (!st && s.req.psi_out) st = gpue_get_wfc(c, s.req.psi_out, GPUE_MEM_HOST, GPUE_C128);
    if (!st && cudaStreamSynchronize(c->stream) != cudaSuccess) st = GPUE_ERR_CUDA;
    gpue_server_result r = make_result(s.req, st ? st : why, s.t_submit, s.t_admit, now_s(S));
    r.steps_done = stopped ? bo.steps : s.steps;
    r.early_stop = stopped ? 1 : 0;
    r.energy = bo.checks > 0 ? bo.energy : NAN;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (r.status == GPUE_ERR_TIMEOUT) S->st.timed_out++;
        if (r.status == GPUE_ERR_CANCELLED) S->st.cancelled++;
        auto it = S->resident_tags.find(s.req.tag);
        if (it != S->resident_tags.end()) S->resident_tags.erase(it);
    }
    return r;
}

// Frees a finished solve's context (cudaFree waits for the device, so this
// runs where the device is idle anyway) and its share of the budget.
void release(gpue_server* S, Solve& s) {
    if (s.c) gpue_ctx_destroy(s.c);
    s.c = nullptr;
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.bytes_resident -= (int64_t)s.bytes;
    S->st.active--;
}

// The results of the solves that left at the last tick, while the next one
// runs (their copies use their own streams); their contexts wait for
// release_zombies.  With release_now (no tick follows) each context is
// freed before its result goes out.
void finish_leaving(gpue_server* S, bool release_now) {
    if (S->leaving.empty()) return;
    const auto tf = std::chrono::steady_clock::now();
    for (Leaving& l : S->leaving) {
        const gpue_server_result r = finish(S, l.s, l.bo, l.stopped, l.why);
        if (release_now) release(S, l.s);
        else S->zombies.push_back(l.s);
        push_result(S, r);
    }
    S->leaving.clear();
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - tf).count();
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.finish_s += dt;
}

void release_zombies(gpue_server* S) {
    if (S->zombies.empty()) return;
    const auto tf = std::chrono::steady_clock::now();
    for (Solve& s : S->zombies) release(S, s);
    S->zombies.clear();
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - tf).count();
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.finish_s += dt;
}

// Enqueues one tick of every resident solve (both runs); returns without
// waiting for the device.
gpue_status tick_issue(gpue_server* S, long& launches, std::string& err) {
    for (int g = 0; g < 2; ++g) S->run[g].members.clear();
    for (size_t i = 0; i < S->active.size(); ++i)
        S->run[S->active[i].req.gstate].members.push_back((int)i);
    launches = 0;
    const auto ti = std::chrono::steady_clock::now();
    for (int g = 0; g < 2; ++g) {
        gpue_status st = issue_run(S, g, S->run[g], launches, err);
        if (st) return st;
    }
    const double issue_s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - ti).count();
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.issue_s += issue_s;
    return GPUE_OK;
}

// Waits for the issued tick and retires the solves that are done.  Solves
// admitted meanwhile (appended to the active list) took no part in it.
gpue_status tick_complete(gpue_server* S, long launches, std::string& err) {
    double busy = 0, pts = 0;
    const Run* first = nullptr;  // the runs overlap: time from the first start
    for (int g = 0; g < 2; ++g) {
        Run& R = S->run[g];
        if (!R.issued) continue;
        if (cudaStreamSynchronize(R.stream) != cudaSuccess) {
            err = std::string("tick: ") + cudaGetErrorString(cudaGetLastError());
            return GPUE_ERR_CUDA;
        }
        if (!first) first = &R;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, first->e0, R.e1);
        busy = std::max(busy, (double)ms * 1e-3);
    }
    // the device is idle: free the contexts whose results went out meanwhile
    release_zombies(S);
    std::vector<char> leave(S->active.size(), 0);
    const auto tf = std::chrono::steady_clock::now();
    std::set<int64_t> cancel;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        cancel.swap(S->cancel);
    }
    const double now = now_s(S);
    for (int g = 0; g < 2; ++g) {
        Run& R = S->run[g];
        if (!R.issued) continue;
        for (size_t k = 0; k < R.members.size(); ++k) {
            Solve& s = S->active[R.members[k]];
            const BatchOut& bo = R.h_outs[k];
            s.steps += S->o.check_steps;
            pts += (double)s.c->N * S->o.check_steps;
            const bool stopped = g == 0 && bo.active == 0;
            gpue_status why = GPUE_OK;
            if (!stopped && s.steps < s.req.max_steps) {
                if (cancel.count(s.req.tag)) why = GPUE_ERR_CANCELLED;
                else if (expired(s.req, s.t_submit, now)) why = GPUE_ERR_TIMEOUT;
            }
            if (stopped || s.steps >= s.req.max_steps || why != GPUE_OK) {
                // its result goes out while the next tick runs
                S->leaving.push_back(Leaving{s, bo, stopped, why});
                leave[R.members[k]] = 1;
                R.drop_graph();  // its arguments name a context leaving the run
            }
        }
    }
    // cancellations of solves admitted during this tick apply after their first
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (size_t i = 0; i < S->active.size(); ++i)
            if ((i >= leave.size() || !leave[i]) && cancel.count(S->active[i].req.tag))
                S->cancel.insert(S->active[i].req.tag);
    }
    std::vector<Solve> keep;
    for (size_t i = 0; i < S->active.size(); ++i)
        if (i >= leave.size() || !leave[i]) keep.push_back(S->active[i]);
    S->active.swap(keep);
    const double finish_s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - tf).count();
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.finish_s += finish_s;
    S->st.ticks++;
    S->st.kernel_launches += launches;
    S->st.point_steps += pts;
    S->st.busy_s += busy;
    return GPUE_OK;
}

void worker_main(gpue_server* S) {
    cudaSetDevice(S->o.device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->active.empty() && S->queue.empty() && S->leaving.empty() &&
                S->zombies.empty())
                S->cv_work.wait_for(lk, std::chrono::milliseconds(20),
                                    [&] { return S->stop || !S->queue.empty(); });
            if (S->stop) return;
        }
        auto timed_admit = [&](bool tune) {
            const auto ta = std::chrono::steady_clock::now();
            admit(S, tune);
            const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() -
                                                            ta).count();
            std::lock_guard<std::mutex> lk(S->mu);
            S->st.admit_s += dt;
        };
        drop_expired(S);
        timed_admit(true);
        if (S->active.empty()) {
            // no tick to overlap: free the last leavers and return them now
            release_zombies(S);
            finish_leaving(S, true);
            continue;
        }
        std::string err;
        long launches = 0;
        gpue_status st = tick_issue(S, launches, err);
        if (!st) finish_leaving(S, false);
        // requests that arrive while the device runs the tick are set up
        // meanwhile (they join the next tick)
        while (!st) {
            timed_admit(false);
            bool busy = false;
            for (Run& R : S->run)
                if (R.issued && cudaStreamQuery(R.stream) == cudaErrorNotReady) busy = true;
            if (!busy) break;
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait_for(lk, std::chrono::microseconds(200),
                                [&] { return S->stop || !S->queue.empty(); });
            if (S->stop) break;
        }
        if (!st) st = tick_complete(S, launches, err);
        if (st) {
            // the device state of every resident solve is now unknown; let
            // whatever was enqueued drain before the contexts are freed
            cudaDeviceSynchronize();
            release_zombies(S);
            finish_leaving(S, true);
            for (Solve& s : S->active) {
                push_result(S, make_result(s.req, st, s.t_submit, s.t_admit, now_s(S)));
                gpue_ctx_destroy(s.c);
            }
            S->active.clear();
            std::lock_guard<std::mutex> lk(S->mu);
            S->broken = true;
            S->err = err;
            S->resident_tags.clear();
            S->cancel.clear();
            S->st.bytes_resident = 0;
            S->st.active = 0;
            while (!S->queue.empty()) {
                const Pending& p = S->queue.front();
                S->done.push_back(make_result(p.req, st, p.t_submit, now_s(S), now_s(S)));
                S->st.failed++;
                S->queue.pop_front();
            }
            S->cv_done.notify_all();
            return;
        }
    }
}

}  // namespace

extern "C" {

const char* gpue_server_last_error(const gpue_server* S) {
    if (!S) return "";
    return S->err.c_str();
}

double gpue_server_clock(const gpue_server* S) { return S ? now_s(S) : 0.0; }

gpue_status gpue_server_create(const gpue_server_opts* opts, gpue_server** out) {
    if (!opts || !out) return GPUE_ERR_INVALID_ARG;
    *out = nullptr;
    const gpue_server_opts& o = *opts;
    if (o.check_steps < 2 || o.check_steps % 2 || o.max_active < 0 || o.hbm_budget_bytes < 0 ||
        (o.precision != GPUE_PREC_FP32 && o.precision != GPUE_PREC_FP64))
        return GPUE_ERR_INVALID_ARG;
    if (cudaSetDevice(o.device) != cudaSuccess) return GPUE_ERR_CUDA;
    std::unique_ptr<gpue_server> S(new gpue_server);
    S->o = o;
    S->t0 = std::chrono::steady_clock::now();
    int64_t budget = o.hbm_budget_bytes;
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return GPUE_ERR_CUDA;
        budget = (int64_t)(0.9 * (double)fr);
    }
    S->st.bytes_budget = budget;
    for (Run& R : S->run) {
        if (cudaStreamCreateWithFlags(&R.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&R.e0) != cudaSuccess || cudaEventCreate(&R.e1) != cudaSuccess ||
            cudaMalloc(&R.nactive, sizeof(int)) != cudaSuccess)
            return GPUE_ERR_CUDA;
    }
    gpue_server* raw = S.get();
    S->worker = std::thread(worker_main, raw);
    *out = S.release();
    return GPUE_OK;
}

gpue_status gpue_server_destroy(gpue_server* S) {
    if (!S) return GPUE_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->worker.joinable()) S->worker.join();
    cudaSetDevice(S->o.device);
    for (Solve& s : S->active)
        if (s.c) gpue_ctx_destroy(s.c);
    for (Leaving& l : S->leaving)
        if (l.s.c) gpue_ctx_destroy(l.s.c);
    for (Solve& s : S->zombies)
        if (s.c) gpue_ctx_destroy(s.c);
    for (Run& R : S->run) {
        if (R.stream) cudaStreamSynchronize(R.stream);
        R.drop_graph();
        R.lanes.destroy();
        R.sink.release();
        if (R.outs) cudaFree(R.outs);
        if (R.h_outs) cudaFreeHost(R.h_outs);
        if (R.nactive) cudaFree(R.nactive);
        if (R.e0) cudaEventDestroy(R.e0);
        if (R.e1) cudaEventDestroy(R.e1);
        if (R.stream) cudaStreamDestroy(R.stream);
    }
    delete S;
    return GPUE_OK;
}

gpue_status gpue_server_submit(gpue_server* S, const gpue_request* q) {
    if (!S || !q || !q->psi0 || (q->gstate != 0 && q->gstate != 1)) return GPUE_ERR_INVALID_ARG;
    const gpue_params& p = q->params;
    if ((p.dimnum != 2 && p.dimnum != 3) || p.yDim != p.xDim ||
        (p.dimnum == 3 && p.zDim != p.xDim))
        return GPUE_ERR_INVALID_ARG;
    if (q->max_steps < S->o.check_steps || q->max_steps % S->o.check_steps)
        return GPUE_ERR_INVALID_ARG;
    if (!gpue_supported_length(S->o.precision, p.xDim)) return GPUE_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->broken) return GPUE_ERR_STATE;
    S->queue.push_back(Pending{*q, now_s(S)});
    S->st.submitted++;
    S->cv_work.notify_all();
    return GPUE_OK;
}

gpue_status gpue_server_cancel(gpue_server* S, int64_t tag) {
    if (!S) return GPUE_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    bool found = false;
    const double now = now_s(S);
    for (auto it = S->queue.begin(); it != S->queue.end();) {
        if (it->req.tag == tag) {
            S->done.push_back(make_result(it->req, GPUE_ERR_CANCELLED, it->t_submit, now, now));
            S->st.failed++;
            S->st.cancelled++;
            it = S->queue.erase(it);
            found = true;
        } else {
            ++it;
        }
    }
    // resident (or being admitted): the worker drops it after the tick in flight
    if (S->resident_tags.count(tag)) {
        S->cancel.insert(tag);
        found = true;
    }
    if (found) S->cv_done.notify_all();
    return found ? GPUE_OK : GPUE_ERR_INVALID_ARG;
}

gpue_status gpue_server_poll(gpue_server* S, gpue_server_result* out, int32_t cap, int32_t* n,
                             double timeout_s) {
    if (!S || !n || cap < 0 || (cap > 0 && !out)) return GPUE_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->done.empty() && timeout_s > 0)
        S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                            [&] { return !S->done.empty(); });
    int k = 0;
    while (k < cap && !S->done.empty()) {
        out[k++] = S->done.front();
        S->done.pop_front();
    }
    *n = k;
    return GPUE_OK;
}

gpue_status gpue_server_get_stats(gpue_server* S, gpue_server_stats* st) {
    if (!S || !st) return GPUE_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    *st = S->st;
    st->queued = (int32_t)S->queue.size();
    return S->broken ? GPUE_ERR_STATE : GPUE_OK;
}

}  // extern "C"
