// vortex.cu -- 2D vortex finder on the resident state (gpue_find_vortices).
//
// GPUE's Tracker::findVortex (src/tracker.cu:102-166) visits the plaquettes
// of a host copy of the state row by row and carries one piece of state
// through the visit: after a marked plaquette, the next in-radius plaquette
// is not marked (its cond_x/cond_y counters).  The marks therefore depend on
// runs: in a run of consecutive candidate plaquettes (visiting order, counting
// only in-radius ones) the 1st, 3rd, 5th ... are marked, and a run starts
// after any in-radius plaquette that is not a candidate.  With r(p) the rank
// of plaquette p among the in-radius plaquettes and r_nc(p) the rank of the
// last non-candidate before it (-1 if none), a candidate is marked iff
// r(p) - r_nc(p) is odd.  Both ranks are prefix counts, so the finder runs as
// five small kernels with no serial walk:
//   k_vtx_winding  one warp per row: candidate code (signed lround of the
//                  winding, 0 for none) per plaquette, in-radius count and
//                  rank of the row's last non-candidate;
//   k_vtx_rows     one warp: row offsets of the ranks and, per row, the rank
//                  of the last non-candidate in the rows before it;
//   k_vtx_mark     one warp per row: ballots give each candidate's ranks; the
//                  marker row is written whole (zeros included);
//   k_vtx_offsets  one warp: offsets of each row's marks in the list, count;
//   k_vtx_list     one warp per row: the marks, in visiting order.
// Every step is integer or comparison work except the winding sum, which
// forms the same IEEE double operations findVortex does (no contraction).

#include "engine_internal.h"

namespace gpue {
namespace {

constexpr double kVPI = 3.141592653589793;  // GPUE's PI (include/constants.h)
constexpr int kRowsPerBlock = 4;               // warps per 128-thread block

__device__ __forceinline__ bool in_radius(const double* x, int i, int j, double radius) {
    const double s = __dadd_rn(__dmul_rn(x[i], x[i]), __dmul_rn(x[j], x[j]));
    return __dsqrt_rn(s) < radius;
}

// Phase of complexScale(complexDiv(a, b), |b|/|a|) (src/minions.cu:62-93),
// wrapped from (-inf, -pi] up by 2 pi as findVortex does.
__device__ __forceinline__ double phase_step(double2 a, double2 b) {
    const double mx = __dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, -b.y));
    const double my = __dadd_rn(__dmul_rn(a.x, -b.y), __dmul_rn(a.y, b.x));
    const double inv = __ddiv_rn(1.0, __dadd_rn(__dmul_rn(b.x, b.x), __dmul_rn(b.y, b.y)));
    const double r = __ddiv_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(b.x, b.x), __dmul_rn(b.y, b.y))),
                               __dsqrt_rn(__dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y))));
    const double gx = __dmul_rn(__dmul_rn(mx, inv), r);
    const double gy = __dmul_rn(__dmul_rn(my, inv), r);
    double d = atan2(gy, gx);
    if (d <= -kVPI) d = __dadd_rn(d, 2 * kVPI);
    return d;
}

template <typename T>
__device__ __forceinline__ double2 load_c(const cx<T>* psi, long g) {
    const cx<T> v = psi[g];
    return make_double2((double)v.x, (double)v.y);
}

// Signed lround(sum / 2 pi) of plaquette (i, j) when |sum| >= 1.9 pi, else 0
// (a NaN sum, from a zero corner, is no candidate, as in findVortex).
template <typename T>
__device__ int plaquette_code(const cx<T>* psi, int n, int i, int j) {
    const double2 c0 = load_c(psi, (long)i * n + j);
    const double2 c1 = load_c(psi, (long)(i + 1) * n + j);
    const double2 c2 = load_c(psi, (long)(i + 1) * n + j + 1);
    const double2 c3 = load_c(psi, (long)i * n + j + 1);
    double sum = __dadd_rn(phase_step(c0, c1), phase_step(c1, c2));
    sum = __dadd_rn(sum, phase_step(c2, c3));
    sum = __dadd_rn(sum, phase_step(c3, c0));
    if (sum >= 1.9 * kVPI || sum <= -1.9 * kVPI) return (int)llround(__ddiv_rn(sum, 2 * kVPI));
    return 0;
}

__device__ __forceinline__ unsigned lanes_below(int lane) { return (1u << lane) - 1u; }

// Rank (within `mask_in`'s lanes) of the highest lane set in `m`, plus base.
__device__ __forceinline__ int rank_of_top(unsigned m, unsigned mask_in, int base) {
    const int top = 31 - __clz(m);
    return base + __popc(mask_in & lanes_below(top));
}

template <typename T>
__global__ void __launch_bounds__(128) k_vtx_winding(const void* psi_, const double* x, int n,
                                                     double radius, signed char* code, int* cnt,
                                                     int* lastnc) {
    const cx<T>* psi = reinterpret_cast<const cx<T>*>(psi_);
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kRowsPerBlock + (threadIdx.x >> 5);
    if (i >= n) return;
    int rank = 0, last = -1;
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int j = j0 + lane;
        const bool inr = i < n - 1 && j < n - 1 && in_radius(x, i, j, radius);
        const int cd = inr ? plaquette_code<T>(psi, n, i, j) : 0;
        if (j < n) code[(long)i * n + j] = (signed char)cd;
        const unsigned mask_in = __ballot_sync(0xffffffffu, inr);
        const unsigned mask_nc = __ballot_sync(0xffffffffu, inr && cd == 0);
        if (mask_nc) last = rank_of_top(mask_nc, mask_in, rank);
        rank += __popc(mask_in);
    }
    if (lane == 0) {
        cnt[i] = rank;
        lastnc[i] = last;
    }
}

// Exclusive prefix over rows by one warp, each lane owning a contiguous
// chunk: rowstart[i] = in-radius plaquettes before row i; carry[i] = global
// rank of the last non-candidate before row i (-1 if none).
__global__ void __launch_bounds__(32) k_vtx_rows(const int* cnt, const int* lastnc, int n,
                                                  int* rowstart, int* carry) {
    const int lane = threadIdx.x;
    const int per = (n + 31) / 32;
    const int lo = min(n, lane * per), hi = min(n, lo + per);
    int s = 0;
    for (int i = lo; i < hi; ++i) s += cnt[i];
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    int run = incl - s;
    int mx = -1;
    for (int i = lo; i < hi; ++i) {
        rowstart[i] = run;
        const int g = lastnc[i] >= 0 ? run + lastnc[i] : -1;
        carry[i] = g;  // this row's own last non-candidate, for now
        mx = max(mx, g);
        run += cnt[i];
    }
    int imax = mx;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, imax, o);
        if (lane >= o) imax = max(imax, v);
    }
    int before = __shfl_up_sync(0xffffffffu, imax, 1);
    if (lane == 0) before = -1;
    for (int i = lo; i < hi; ++i) {
        const int g = carry[i];
        carry[i] = before;
        before = max(before, g);
    }
}

__global__ void __launch_bounds__(128) k_vtx_mark(const signed char* code, const double* x, int n,
                                                  double radius, const int* rowstart,
                                                  const int* carry, int* marker, int* rowfound) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kRowsPerBlock + (threadIdx.x >> 5);
    if (i >= n) return;
    int rank = rowstart[i], nc = carry[i], found = 0;
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int j = j0 + lane;
        const bool inr = i < n - 1 && j < n - 1 && in_radius(x, i, j, radius);
        const int cd = inr ? (int)code[(long)i * n + j] : 0;
        const unsigned mask_in = __ballot_sync(0xffffffffu, inr);
        const unsigned mask_nc = __ballot_sync(0xffffffffu, inr && cd == 0);
        bool mark = false;
        if (cd != 0) {
            const unsigned before = mask_nc & lanes_below(lane);
            const int r_nc = before ? rank_of_top(before, mask_in, rank) : nc;
            const int r = rank + __popc(mask_in & lanes_below(lane));
            mark = ((r - r_nc) & 1) != 0;
        }
        if (j < n) marker[(long)i * n + j] = mark ? (cd < 0 ? -cd : cd) : 0;
        found += __popc(__ballot_sync(0xffffffffu, mark));
        if (mask_nc) nc = rank_of_top(mask_nc, mask_in, rank);
        rank += __popc(mask_in);
    }
    if (lane == 0) rowfound[i] = found;
}

__global__ void __launch_bounds__(32) k_vtx_offsets(const int* rowfound, int n, int* rowoff,
                                                     int* found) {
    const int lane = threadIdx.x;
    const int per = (n + 31) / 32;
    const int lo = min(n, lane * per), hi = min(n, lo + per);
    int s = 0;
    for (int i = lo; i < hi; ++i) s += rowfound[i];
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    int run = incl - s;
    for (int i = lo; i < hi; ++i) {
        rowoff[i] = run;
        run += rowfound[i];
    }
    if (lane == 31) *found = incl;
}

__global__ void __launch_bounds__(128) k_vtx_list(const int* marker, const signed char* code,
                                                  const int* rowfound, const int* rowoff, int n,
                                                  gpue_vortex* list, int cap) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * kRowsPerBlock + (threadIdx.x >> 5);
    if (i >= n || rowfound[i] == 0) return;
    int idx = rowoff[i];
    for (int j0 = 0; j0 < n && idx < cap; j0 += 32) {
        const int j = j0 + lane;
        const int m = j < n ? marker[(long)i * n + j] : 0;
        const unsigned mask = __ballot_sync(0xffffffffu, m != 0);
        const int k = idx + __popc(mask & lanes_below(lane));
        if (m != 0 && k < cap) {
            gpue_vortex v;
            v.i = i;
            v.j = j;
            v.marker = m;
            v.winding = code[(long)i * n + j];
            list[k] = v;
        }
        idx += __popc(mask);
    }
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace
}  // namespace gpue

using namespace gpue_eng;

gpue_status gpue_find_vortices(gpue_ctx* c, double radius, int32_t* marker, int32_t mem,
                               gpue_vortex* list, int32_t cap, int32_t* found) {
    if (!c) return GPUE_ERR_INVALID_ARG;
    if (mem != GPUE_MEM_HOST && mem != GPUE_MEM_DEVICE)
        return fail(c, GPUE_ERR_INVALID_ARG, "mem must be GPUE_MEM_HOST or GPUE_MEM_DEVICE");
    if (cap < 0 || (cap > 0 && !list))
        return fail(c, GPUE_ERR_INVALID_ARG, "list capacity %d without a list", cap);
    if (c->dim != 2) return fail(c, GPUE_ERR_UNSUPPORTED, "the vortex finder is 2D only");
    if (!c->have_wfc) return fail(c, GPUE_ERR_STATE, "no wavefunction set");
    CK(cudaSetDevice(c->device));
    const int sp = c->polished ? GPUE_PREC_FP64 : c->prec;
    const int gs = c->tab[sp].built_for < 0 ? 0 : c->tab[sp].built_for;
    gpue_status st = build_tables(c, sp, gs);
    if (st) return st;
    st = apply_pending_scale(c, sp);
    if (st) return st;

    const int n = c->ax[0].n;
    const long N = (long)n * n;
    const long list_cap_ws = N / 2 + 1;  // marks never follow one another: at most ceil(N'/2)
    const size_t b_code = align256((size_t)N);
    const size_t b_rows = align256(sizeof(int) * (6 * (size_t)n + 1));
    const size_t b_marker = align256(sizeof(int) * (size_t)N);
    const size_t b_list = align256(sizeof(gpue_vortex) * (size_t)list_cap_ws);
    const size_t need = b_code + b_rows + b_marker + b_list;
    if (c->vtx_ws_bytes < need) {
        if (c->vtx_ws) CK(cudaFree(c->vtx_ws));
        c->vtx_ws = nullptr;
        c->vtx_ws_bytes = 0;
        CK(cudaMalloc(&c->vtx_ws, need));
        c->vtx_ws_bytes = need;
    }
    unsigned char* w = (unsigned char*)c->vtx_ws;
    signed char* code = (signed char*)w;
    int* rows = (int*)(w + b_code);
    int *cnt = rows, *lastnc = rows + n, *rowstart = rows + 2 * n, *carry = rows + 3 * n,
        *rowfound = rows + 4 * n, *rowoff = rows + 5 * n, *dfound = rows + 6 * n;
    int* dmarker = (mem == GPUE_MEM_DEVICE && marker) ? marker : (int*)(w + b_code + b_rows);
    const bool dev_list = mem == GPUE_MEM_DEVICE && list;
    gpue_vortex* dlist =
        dev_list ? list : (gpue_vortex*)(w + b_code + b_rows + b_marker);
    const int dcap = dev_list ? cap : (int)std::min<long>(cap, list_cap_ws);

    const double* x = c->tab[sp].pos[0];
    const void* psi = state_of(c, sp);
    const int blocks = (n + kRowsPerBlock - 1) / kRowsPerBlock;
    if (sp == GPUE_PREC_FP32)
        k_vtx_winding<float><<<blocks, 128, 0, c->stream>>>(psi, x, n, radius, code, cnt, lastnc);
    else
        k_vtx_winding<double><<<blocks, 128, 0, c->stream>>>(psi, x, n, radius, code, cnt, lastnc);
    k_vtx_rows<<<1, 32, 0, c->stream>>>(cnt, lastnc, n, rowstart, carry);
    k_vtx_mark<<<blocks, 128, 0, c->stream>>>(code, x, n, radius, rowstart, carry, dmarker,
                                              rowfound);
    k_vtx_offsets<<<1, 32, 0, c->stream>>>(rowfound, n, rowoff, dfound);
    if (list && dcap > 0)
        k_vtx_list<<<blocks, 128, 0, c->stream>>>(dmarker, code, rowfound, rowoff, n, dlist,
                                                  dcap);
    CK(cudaGetLastError());
    int h_found = 0;
    CK(cudaMemcpyAsync(&h_found, dfound, sizeof h_found, cudaMemcpyDeviceToHost, c->stream));
    if (marker && mem == GPUE_MEM_HOST)
        CK(cudaMemcpyAsync(marker, dmarker, sizeof(int) * (size_t)N, cudaMemcpyDeviceToHost,
                           c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (list && !dev_list && cap > 0) {
        const int k = std::min(h_found, dcap);
        if (k > 0)
            CK(cudaMemcpy(list, dlist, sizeof(gpue_vortex) * (size_t)k, cudaMemcpyDeviceToHost));
    }
    if (found) *found = h_found;
    return GPUE_OK;
}
