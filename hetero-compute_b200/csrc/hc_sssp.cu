// Single-source shortest paths as one persistent cooperative launch per source.
//
// Reference path: sssp_pull_gpu (src/kernels/gpu/sssp.cuh:42-100) sweeps every
// vertex each epoch with an in-place Bellman-Ford pull over float weights and
// round-trips a counter to the host per epoch.  Here the epoch loop stays on
// the device and each epoch picks its direction:
//   push  relax only the edges out of vertices whose distance dropped (int32
//         atomicMin), split near/far by a moving threshold (Davidson et al.,
//         "Work-efficient parallel GPU methods for single-source shortest
//         paths", IPDPS 2014);
//   pull  when the frontier's edges exceed M / pull_alpha, sweep every row
//         with the reference's own Bellman-Ford pull (min over neighbours of
//         dist[u] + w) over each row's (neighbour, weight) pairs in weight
//         order, stopping a row once no later pair can lower it, without
//         per-edge atomics, then turn the vertices it lowered back into the
//         near queue / far pile.
// Distances are exact integers; unreachable = INT32_MAX.
//
// Working set (N vertices): dist int32[N]; near queues q[2] int32[N];
// far piles far[2] int32[N]; stamp / fstamp int32[N] (queue dedup without
// clearing: a vertex joins the epoch-E queue by raising stamp[v] to E);
// changed bitmap uint32[N/32] (pull sweeps); tasks int2[] for long rows.
// Per graph: the pull sweeps' pair array int2[M + 64] (weight_order_rows).
#include <algorithm>
#include <climits>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <vector>

#include "hc_expand.cuh"
#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr int kSsspThreads = 512;
constexpr int kPullThreads = 256;
constexpr int kTraceEpochs = 96;
constexpr int kDefaultPullAlpha = 10;
// After a pull epoch, far piles of at most this many entries end the near/far
// phases (one last phase takes every remaining vertex).
#ifndef HC_SSSP_TAIL_PILE
#define HC_SSSP_TAIL_PILE 16384
#endif
constexpr int kTailPile = HC_SSSP_TAIL_PILE;

struct SsspCtl {
    GridSync gs;
    // Pull epochs run as a separate kernel (sssp_pull_kernel): the persistent
    // kernel saves its loop state here and exits with need_pull set, and the
    // next launch (resume set) folds the lowered rows into its queues.
    int need_pull, resume;
    int finished;  // the run is over: later launches of the chain return at once
    int saved_E, saved_phase, saved_pulls, saved_T;
    int saved_fgen;  // the far-pile claim the resumed launch uses
    unsigned long long t_start;
    int qlen[3];
    int tasks[3];
    unsigned long long mf[3];  // degree sum of each near queue
    int far_len[2];
    int min_far;
    int epochs, phases, pulls;
    unsigned long long vproc, erelax;
    // Degree sum of the rows a pull sweep lowered below the near threshold:
    // the next epoch's push-or-pull test, without building its queue.
    unsigned long long pull_mf;
    struct {
        int nq, phase;
        unsigned long long t_ns;
    } trace[kTraceEpochs + 1];  // per-epoch record for HC_TRACE=1 (phase < 0: pull sweep)
};

struct SsspArgs {
    const int64_t *index;
    const int32_t *nbr;
    const int32_t *w;
    int32_t n, n_active;
    int64_t m;
    int32_t *dist;
    int32_t *q0, *q1, *far0, *far1, *stamp, *fstamp;
    uint32_t *changed;
    int2 *tasks;
    SsspCtl *ctl;
    PrPlanDev plan;
    const int2 *adj;  // pull sweeps: (neighbour, weight) pairs of each row in weight-bucket order
    int ws;           // bucket shift: bucket(w) = w >> ws < 256
    int32_t src;
    int32_t delta;  // <= 0: no far pile (plain frontier Bellman-Ford)
    int pull_alpha;  // <= 0: push only
    int max_epochs;
};

// dist + w for a distance and a weight in [0, INT32_MAX], clamped at
// INT32_MAX (unreachable): the sum never wraps, and a candidate that reaches
// the clamp lowers nothing.  Callers check afterwards that no distance came
// within the largest weight of the clamp.
__device__ __forceinline__ int32_t sat_add(int32_t d, int32_t w) {
    const uint32_t s = (uint32_t)d + (uint32_t)w;
    return s < (uint32_t)kInfDist ? (int32_t)s : kInfDist;
}

// Push relaxation visitor: nd = dist[u] + w; lower dist[v] with atomicMin and
// queue v once per epoch (near) or once per phase (far), by raising a stamp.
struct RelaxVisit {
    const int64_t *index;
    const int32_t *nbr, *w;
    int32_t *dist, *stamp, *fstamp;
    int32_t *qnext;
    int *qlen;
    int32_t *fpile;
    int *fpile_len;
    int32_t T;
    int next_e, far_claim;
    bool use_far;
    unsigned long long relaxed;
    unsigned long long mf;  // degree sum of this thread's near appends
    struct Item {
        int32_t v, nd, dv;
    };
    __device__ __forceinline__ void load(Item &it, int32_t u, int64_t e) {
        it.v = nbr[e];
        it.nd = sat_add(__ldcg(dist + u), w[e]);
    }
    __device__ __forceinline__ void probe(Item &it) { it.dv = __ldcg(dist + it.v); }
    // Stages across the round's items: all atomicMins in flight, then all
    // stamp claims, then one append per queue for the whole warp.
    __device__ __forceinline__ void commit(Item (&it)[kUnroll], const bool (&act)[kUnroll]) {
        bool imp[kUnroll], near[kUnroll], far[kUnroll];
        int32_t prev[kUnroll], old[kUnroll], v[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; j++) {
            relaxed += act[j];
            imp[j] = act[j] && it[j].nd < it[j].dv;
            prev[j] = imp[j] ? atomicMin(dist + it[j].v, it[j].nd) : 0;
        }
#pragma unroll
        for (int j = 0; j < kUnroll; j++) {
            imp[j] = imp[j] && it[j].nd < prev[j];
            const bool is_near = it[j].nd < T;
            old[j] = imp[j] ? (is_near ? atomicMax(stamp + it[j].v, next_e) : atomicMax(fstamp + it[j].v, far_claim))
                            : 0;
        }
#pragma unroll
        for (int j = 0; j < kUnroll; j++) {
            const bool is_near = it[j].nd < T;
            near[j] = imp[j] && is_near && old[j] < next_e;
            far[j] = imp[j] && !is_near && old[j] < far_claim;
            v[j] = imp[j] ? it[j].v : 0;
            if (near[j]) mf += (unsigned long long)(index[v[j] + 1] - index[v[j]]);
        }
        warp_append_n(near, v, qnext, qlen);
        if (use_far) warp_append_n(far, v, fpile, fpile_len);
    }
};

// Weight buckets of the pull sweeps' pair array: bucket(w) = w >> ws, ws the
// shift that brings the largest weight below 256, non-decreasing along each
// row.  Every pair at or after one of bucket b has weight >= b << ws.
__device__ __forceinline__ int wbucket(int32_t w, int ws) { return w >> ws; }
__device__ __forceinline__ int32_t wbucket_floor(int bk, int ws) { return bk << ws; }

// dist[u] + w for a pair whose weight is below `bound`, else INT32_MAX
// without touching dist: a candidate is at least its weight, so a pair with
// w >= bound cannot lower a row whose best so far is `bound`.
// The gather goes through L1 (.ca): most edges point at a few thousand hub
// rows, whose distances then stay on the SM.  A value cached earlier in the
// same sweep can be stale, but distances only fall, so it is an upper bound,
// and the row that lowered it is marked changed and relaxed again next epoch;
// kernel boundaries and the grid barrier's fence invalidate L1 between epochs.
__device__ __forceinline__ int32_t pull_cand(const SsspArgs &a, int2 p, int32_t bound) {
    return p.y < bound ? sat_add(__ldca(a.dist + p.x), p.y) : kInfDist;
}

// One Bellman-Ford pull over every row with edges (the reference's epoch,
// src/kernels/gpu/sssp.cuh:120-281), on the shared row plan, over the rows'
// pairs in weight-bucket order.  Hub chunks and long rows walk their range
// 128 pairs at a time with a running bound (the row's distance, then the best
// candidate): pairs at or above it gather nothing, and the walk stops at the
// first window whose leading bucket floor reaches it.  They lower dist by
// atomicMin.  Stream groups (32 rows, one warp) read every pair, gather only
// those below their row's bound and keep each row's minimum in shared memory;
// they own their rows and their changed-bitmap word.  Lowered vertices are marked
// in `changed`.
template <bool kStats>
__device__ __forceinline__ void pull_sweep(const SsspArgs &a, int gwarp, int nwarps, int32_t (*s_acc)[32],
                                           unsigned long long &my_e, int32_t T, unsigned long long &my_mf) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const PrPlanDev &p = a.plan;
    const int total = p.n_tasks + p.n_long + p.n_stream;
    for (int item = gwarp; item < total; item += nwarps) {
        if (item < p.n_tasks + p.n_long) {
            int32_t r;
            int64_t b, e;
            // The leading weight of the next window, read one window ahead so
            // that the stop test comes before the window's loads.  A long row
            // always takes its first window; a hub row's later chunk tests its
            // first one too (it starts among the row's heavier pairs).
            const int32_t *wcol = reinterpret_cast<const int32_t *>(a.adj) + 1;
            bool test_first = false;
            if (item < p.n_tasks) {
                const int2 tk = p.tasks[item];
                r = p.hubs[tk.x].row;
                const int64_t rb = a.index[r], re = a.index[r + 1];
                b = rb + (int64_t)tk.y * kHubChunk;
                e = min(re, b + (int64_t)kHubChunk);
                test_first = tk.y > 0;
            } else {
                r = p.longrows[item - p.n_tasks];
                b = a.index[r];
                e = a.index[r + 1];
            }
            int32_t wnext = test_first ? wcol[2 * b] : 0;
            const int32_t d0 = __shfl_sync(kFull, __ldcg(a.dist + r), 0);
            int32_t bound = d0;
            int64_t i0 = b;
            for (; i0 < e; i0 += 128) {
                // Pair i0 carries the smallest bucket of the rest of the range.
                if ((i0 > b || test_first) && wbucket_floor(wbucket(wnext, a.ws), a.ws) >= bound) break;
                int2 q[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int64_t i = i0 + 32 * j + lane;
                    q[j] = i < e ? a.adj[i] : make_int2(0, kInfDist);
                }
                if (i0 + 128 < e) wnext = wcol[2 * (i0 + 128)];
                int32_t m = kInfDist;
#pragma unroll
                for (int j = 0; j < 4; j++) m = min(m, pull_cand(a, q[j], bound));
                bound = min(bound, warp_min(m));
            }
            if (lane == 0) {
                if (bound < d0 && bound < __ldcg(a.dist + r) && bound < atomicMin(a.dist + r, bound)) {
                    const uint32_t bit = 1u << (r & 31);
                    if (!(atomicOr(a.changed + (r >> 5), bit) & bit) && bound < T)
                        my_mf += (unsigned long long)(a.index[r + 1] - a.index[r]);
                }
                if (kStats) my_e += (unsigned long long)(min(i0, e) - b);
            }
        } else {
            const int32_t r0 = p.stream[item - p.n_tasks - p.n_long] * 32;
            const int32_t r = r0 + lane;
            const int32_t rc = min(r, a.n_active);
            const int64_t s0 = a.index[r0];
            const int32_t rel = (int32_t)(a.index[rc] - s0);
            const int32_t gend = (int32_t)(a.index[min(r0 + 32, a.n_active)] - s0);
            // This lane's row: its distance at the start, then the best found.
            int32_t rbound = r < a.n_active ? __ldcg(a.dist + r) : kInfDist;
            const int32_t rd0 = rbound;
            s_acc[wib][lane] = kInfDist;
            __syncwarp();
            // Four 32-pair chunks per pass: the pair loads go out first, then
            // each pair finds its row among the group's offsets, then the
            // gathers below the row's bound.
            for (int k0 = 0; k0 < gend; k0 += 128) {
                int2 q[4];
                int owner[4];
                int32_t vals[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int k = k0 + 32 * j + lane;
                    q[j] = k < gend ? a.adj[s0 + k] : make_int2(0, kInfDist);
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int k = k0 + 32 * j + lane;
                    int lo = 0;
#pragma unroll
                    for (int st = 16; st > 0; st >>= 1) {
                        const int c = __shfl_sync(kFull, rel, lo + st);
                        if (c <= k) lo += st;
                    }
                    owner[j] = k < gend ? lo : 32;
                    const int32_t ob = __shfl_sync(kFull, rbound, lo);
                    vals[j] = pull_cand(a, q[j], ob);
                }
                // Most pairs sit at or above their row's bound and bring no
                // candidate: the few that do go to the row's slot by a
                // shared-memory atomic minimum.
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (vals[j] < kInfDist) atomicMin(&s_acc[wib][owner[j]], vals[j]);
                __syncwarp();
                rbound = min(rbound, s_acc[wib][lane]);
            }
            bool ch = false;
            const int32_t rnext = __shfl_down_sync(kFull, rel, 1);
            if (r < a.n_active && rbound < rd0 && rbound < __ldcg(a.dist + r)) {
                a.dist[r] = rbound;  // the group is the only writer of its rows
                ch = true;
                if (rbound < T) my_mf += (unsigned long long)((lane == 31 ? gend : rnext) - rel);
            }
            const unsigned bal = __ballot_sync(kFull, ch);
            if (lane == 0) {
                if (bal) a.changed[r0 >> 5] = bal;
                if (kStats) my_e += (unsigned long long)gend;
            }
            __syncwarp();
        }
    }
}

template <bool kStats>
__global__ void __launch_bounds__(kSsspThreads, 2) sssp_persistent(SsspArgs a) {
    __shared__ unsigned long long s_red[32];
    __shared__ int s_min[32];
    __shared__ uint32_t s_fold[kSsspThreads / 32][2][32];  // per warp: near / far masks of its 32 words
    SsspCtl *ctl = a.ctl;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthreads = gridDim.x * blockDim.x;
    const int gwarp = gtid >> 5, nwarps = nthreads >> 5;
    const int lane = threadIdx.x & 31;
    const int W_act = (a.n_active + 31) >> 5;

    const bool use_far = a.delta > 0;
    int32_t T = use_far ? a.delta : kInfDist;
    int E = 0, phase = 0, pulls = 0;
    // Far-pile claim: a vertex is in the current pile when fstamp[v] == fgen.
    int fgen = 1;
    unsigned long long my_v = 0, my_e = 0;
    // Every block reads the same control words (written before this launch).
    if (__ldcg(&ctl->finished) || __ldcg(&ctl->gs.err)) return;  // a speculative launch past the end
    const bool resumed = __ldcg(&ctl->resume) != 0;
    unsigned long long t_start;
    unsigned long long pull_mf = 0;  // read before the barrier below; block 0 may reset it after
    if (!resumed) {
        for (int i = gtid; i < a.n; i += nthreads) {
            a.dist[i] = kInfDist;
            a.stamp[i] = -1;
            a.fstamp[i] = -1;
        }
        for (int i = gtid; i < W_act; i += nthreads) a.changed[i] = 0;
        t_start = globaltimer_ns();
        if (gtid == 0) ctl->t_start = t_start;
        if (!grid_barrier(&ctl->gs)) return;
        if (gtid == 0) {
            a.dist[a.src] = 0;
            a.stamp[a.src] = 0;
            a.q0[0] = a.src;
            ctl->qlen[0] = 1;
            ctl->mf[0] = (unsigned long long)(a.index[a.src + 1] - a.index[a.src]);
            ctl->min_far = kInfDist;
        }
        if (!grid_barrier(&ctl->gs)) return;
    } else {
        E = __ldcg(&ctl->saved_E);
        phase = __ldcg(&ctl->saved_phase);
        pulls = __ldcg(&ctl->saved_pulls);
        T = __ldcg(&ctl->saved_T);
        fgen = __ldcg(&ctl->saved_fgen);
        pull_mf = __ldcg(&ctl->pull_mf);
        t_start = __ldcg(&ctl->t_start);
        if (!grid_barrier(&ctl->gs)) return;  // everyone has read the saved state
        if (gtid == 0) ctl->need_pull = 0;
    }
    bool after_pull = resumed;  // epoch E's pull sweep ran in sssp_pull_kernel

    for (;;) {
        const int cur = E % 3, nxt = (E + 1) % 3, old = (E + 2) % 3;
        int32_t *qcur = (E & 1) ? a.q1 : a.q0;
        int32_t *qnext = (E & 1) ? a.q0 : a.q1;
        const int next_e = E + 1;
        if (after_pull) {
            after_pull = false;
            // When the rows the pull lowered already make the next epoch a
            // pull, that sweep propagates their values anyway: clear the
            // changed bitmap and hand over at once, without queueing them.
            if (a.pull_alpha > 0 && (double)pull_mf * (double)a.pull_alpha > (double)a.m && E + 1 < a.max_epochs) {
                for (int w = gtid; w < W_act; w += nthreads) a.changed[w] = 0;
                E++;
                if (gtid == 0) {
                    const int old_slot = (E + 2) % 3;
                    ctl->qlen[old_slot] = 0;
                    ctl->tasks[old_slot] = 0;
                    ctl->mf[old_slot] = 0;
                    if (E < kTraceEpochs) {
                        ctl->trace[E].nq = 0;
                        ctl->trace[E].phase = -1 - phase;
                        ctl->trace[E].t_ns = globaltimer_ns();
                    }
                    ctl->saved_E = E;
                    ctl->saved_phase = phase;
                    ctl->saved_pulls = pulls + 1;
                    ctl->saved_T = T;
                    ctl->saved_fgen = fgen + 1;
                    ctl->pull_mf = 0;
                    ctl->resume = 1;
                    ctl->need_pull = 1;
                }
                break;
            }
            int32_t *fpile = (phase & 1) ? a.far1 : a.far0;
            int *fpile_len = &ctl->far_len[phase & 1];
            // Lowered vertices back into the near queue / far pile.  A warp
            // takes 32 words of the changed bitmap; pass 1 classifies their
            // vertices a word at a time (lane l takes vertex 32j + l of word j:
            // coalesced reads; each vertex is in one bit, so its stamps need
            // no atomics) and keeps the ballots in shared memory; pass 2
            // writes the queue and pile entries at offsets taken with one
            // atomicAdd per warp.
            unsigned long long mf_next = 0;
            const int wib = threadIdx.x >> 5;
            const uint32_t below = (1u << lane) - 1u;
            for (int w0 = gwarp * 32; w0 < W_act; w0 += nwarps * 32) {
                const int w = w0 + lane;
                uint32_t bits = 0;
                if (w < W_act) {
                    bits = __ldcg(a.changed + w);
                    if (bits) a.changed[w] = 0;
                }
                const unsigned words = __ballot_sync(kFull, bits != 0u);
                int n_near = 0, n_far = 0;
                // Four words per round, their loads issued together.
                for (unsigned left = words; left;) {
                    int j[4];
                    bool mine[4];
                    int32_t d[4], sp[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        j[k] = left ? __ffs(left) - 1 : -1;
                        if (left) left &= left - 1u;
                        const uint32_t word = __shfl_sync(kFull, bits, j[k] < 0 ? 0 : j[k]);
                        mine[k] = j[k] >= 0 && ((word >> lane) & 1u);
                        d[k] = mine[k] ? __ldcg(a.dist + (w0 + j[k]) * 32 + lane) : 0;
                    }
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const int32_t v = (w0 + j[k]) * 32 + lane;
                        sp[k] = !mine[k] ? 0 : d[k] < T ? a.stamp[v] : a.fstamp[v];
                    }
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const int32_t v = (w0 + j[k]) * 32 + lane;
                        bool near = false, far = false;
                        if (mine[k]) {
                            if (d[k] < T) {
                                near = sp[k] < next_e;
                                if (near) a.stamp[v] = next_e;
                            } else {
                                far = sp[k] < fgen;
                                if (far) a.fstamp[v] = fgen;
                            }
                            if (near) mf_next += (unsigned long long)(a.index[v + 1] - a.index[v]);
                        }
                        const uint32_t nm = __ballot_sync(kFull, near), fm = __ballot_sync(kFull, far);
                        if (lane == 0 && j[k] >= 0) {
                            s_fold[wib][0][j[k]] = nm;
                            s_fold[wib][1][j[k]] = fm;
                        }
                        n_near += __popc(nm);
                        n_far += __popc(fm);
                    }
                }
                if (!use_far) n_far = 0;
                int nbase = 0, fbase = 0;
                if (lane == 0) {
                    if (n_near) nbase = atomicAdd(&ctl->qlen[nxt], n_near);
                    if (n_far) fbase = atomicAdd(fpile_len, n_far);
                }
                nbase = __shfl_sync(kFull, nbase, 0);
                fbase = __shfl_sync(kFull, fbase, 0);
                __syncwarp();
                for (unsigned left = words; left;) {
                    const int j = __ffs(left) - 1;
                    left &= left - 1u;
                    const uint32_t nm = s_fold[wib][0][j], fm = use_far ? s_fold[wib][1][j] : 0u;
                    const int32_t v = (w0 + j) * 32 + lane;
                    if ((nm >> lane) & 1u) qnext[nbase + __popc(nm & below)] = v;
                    if ((fm >> lane) & 1u) fpile[fbase + __popc(fm & below)] = v;
                    nbase += __popc(nm);
                    fbase += __popc(fm);
                }
                __syncwarp();
            }
            mf_next = block_sum(mf_next, s_red);
            if (threadIdx.x == 0 && mf_next) atomicAdd(&ctl->mf[nxt], mf_next);
            if (!grid_barrier(&ctl->gs)) return;
            E++;
            continue;
        }
        if (gtid == 0 && globaltimer_ns() - t_start > c_limits.run_ns) atomicExch(&ctl->gs.err, (int)HC_ERR_TIMEOUT);
        int nq = __ldcg(&ctl->qlen[cur]);
        if (nq == 0) {
            if (!use_far) break;
            int32_t *fcur = (phase & 1) ? a.far1 : a.far0;
            int32_t *fnew = (phase & 1) ? a.far0 : a.far1;
            const int fl = __ldcg(&ctl->far_len[phase & 1]);
            if (fl == 0) break;
            // Smallest live distance in the far pile picks the next bucket.
            int mn = kInfDist;
            for (int i = gtid; i < fl; i += nthreads) {
                const int32_t d = __ldcg(a.dist + __ldcg(fcur + i));
                if (d >= T) mn = min(mn, d);
            }
            mn = warp_min(mn);
            if (lane == 0) s_min[threadIdx.x >> 5] = mn;
            __syncthreads();
            if (threadIdx.x < 32) {
                int x = threadIdx.x < (blockDim.x >> 5) ? s_min[threadIdx.x] : kInfDist;
                x = warp_min(x);
                if (threadIdx.x == 0 && x < kInfDist) atomicMin(&ctl->min_far, x);
            }
            if (!grid_barrier(&ctl->gs)) return;
            const int32_t mfar = __ldcg(&ctl->min_far);
            if (mfar == kInfDist) break;
            const int32_t T_old = T;
            // After a pull sweep (the dense part of a small-diameter graph is
            // done) a small pile is finished in one last near phase: a phase
            // costs a few grid barriers however few vertices it holds, and
            // relaxing those few out of distance order costs little.  On a
            // high-diameter graph (no pulls) the pile is the thin wavefront
            // and keeps its distance order.
            const long long tn = pulls > 0 && fl <= kTailPile
                                     ? (long long)kInfDist
                                     : ((long long)mfar / a.delta + 1) * (long long)a.delta;
            T = (int32_t)(tn < (long long)kInfDist ? tn : (long long)kInfDist);
            // Split: [T_old, T) joins the epoch-E queue, >= T stays far.  A
            // warp takes 1024 consecutive pile entries: pass 1 classifies them
            // 32 at a time and keeps the ballots in shared memory, pass 2
            // writes them at offsets taken with one atomicAdd per warp.
            unsigned long long mf_split = 0;
            const int wib = threadIdx.x >> 5;
            const uint32_t below = (1u << lane) - 1u;
            // Rounds of 32 entries per warp chunk: enough for every warp to
            // get one chunk, at most 32 (the shared ballot slots).
            const int per = min(32, max(1, (fl + 32 * nwarps - 1) / (32 * nwarps)));
            for (int c0 = gwarp * 32 * per; c0 < fl; c0 += nwarps * 32 * per) {
                const int rounds = min(per, (fl - c0 + 31) / 32);
                int n_near = 0, n_far = 0;
                for (int j0 = 0; j0 < rounds; j0 += 4) {
                    int32_t v[4], d[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const int i = c0 + 32 * (j0 + k) + lane;
                        v[k] = (j0 + k < rounds && i < fl) ? __ldcg(fcur + i) : -1;
                    }
#pragma unroll
                    for (int k = 0; k < 4; k++) d[k] = v[k] >= 0 ? __ldcg(a.dist + v[k]) : 0;
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        bool to_near = false, to_far = false;
                        if (v[k] >= 0) {
                            if (d[k] >= T_old && d[k] < T) to_near = atomicMax(a.stamp + v[k], E) < E;
                            else if (d[k] >= T) to_far = atomicMax(a.fstamp + v[k], fgen + 1) < fgen + 1;
                            if (to_near) mf_split += (unsigned long long)(a.index[v[k] + 1] - a.index[v[k]]);
                        }
                        const uint32_t nm = __ballot_sync(kFull, to_near), fm = __ballot_sync(kFull, to_far);
                        if (lane == 0 && j0 + k < rounds) {
                            s_fold[wib][0][j0 + k] = nm;
                            s_fold[wib][1][j0 + k] = fm;
                        }
                        n_near += __popc(nm);
                        n_far += __popc(fm);
                    }
                }
                int nbase = 0, fbase = 0;
                if (lane == 0) {
                    if (n_near) nbase = atomicAdd(&ctl->qlen[cur], n_near);
                    if (n_far) fbase = atomicAdd(&ctl->far_len[(phase + 1) & 1], n_far);
                }
                nbase = __shfl_sync(kFull, nbase, 0);
                fbase = __shfl_sync(kFull, fbase, 0);
                __syncwarp();
                for (int j = 0; j < rounds; j++) {
                    const uint32_t nm = s_fold[wib][0][j], fm = s_fold[wib][1][j];
                    if ((nm | fm) >> lane & 1u) {
                        const int32_t v = __ldcg(fcur + c0 + 32 * j + lane);
                        if ((nm >> lane) & 1u) qcur[nbase + __popc(nm & below)] = v;
                        else fnew[fbase + __popc(fm & below)] = v;
                    }
                    nbase += __popc(nm);
                    fbase += __popc(fm);
                }
                __syncwarp();
            }
            mf_split = block_sum(mf_split, s_red);
            if (threadIdx.x == 0 && mf_split) atomicAdd(&ctl->mf[cur], mf_split);
            if (!grid_barrier(&ctl->gs)) return;
            if (gtid == 0) {
                ctl->far_len[phase & 1] = 0;
                ctl->min_far = kInfDist;
            }
            phase++;
            fgen++;
            nq = __ldcg(&ctl->qlen[cur]);
            if (nq == 0) continue;
        }
        if (E >= a.max_epochs) {
            if (gtid == 0) atomicExch(&ctl->gs.err, (int)HC_ERR_NOT_CONVERGED);
            break;
        }
        if (gtid == 0) {
            ctl->qlen[old] = 0;
            ctl->tasks[old] = 0;
            ctl->mf[old] = 0;
        }
        // After the far split above: `phase` may have advanced.
        int32_t *fpile = (phase & 1) ? a.far1 : a.far0;
        int *fpile_len = &ctl->far_len[phase & 1];
        const unsigned long long mfc = __ldcg(&ctl->mf[cur]);
        const bool pull = a.pull_alpha > 0 && (double)mfc * (double)a.pull_alpha > (double)a.m;
        if (gtid == 0 && E < kTraceEpochs) {
            ctl->trace[E].nq = nq;
            ctl->trace[E].phase = pull ? -1 - phase : phase;
            ctl->trace[E].t_ns = globaltimer_ns();
        }
        if (kStats && gtid == 0) my_v += nq;
        if (pull) {
            // Hand the epoch to sssp_pull_kernel and resume after it.
            if (gtid == 0) {
                ctl->saved_E = E;
                ctl->saved_phase = phase;
                ctl->saved_pulls = pulls + 1;
                ctl->saved_T = T;
                // The pull sweep propagates every distance it starts from, so
                // the pull launch empties the far pile; the rows it lowers
                // rejoin under a new claim.
                ctl->saved_fgen = fgen + 1;
                ctl->pull_mf = 0;
                ctl->resume = 1;
                ctl->need_pull = 1;
            }
            break;
        } else {
            RelaxVisit relax{a.index, a.nbr, a.w, a.dist, a.stamp, a.fstamp, qnext, &ctl->qlen[nxt], fpile,
                             fpile_len, T, next_e, fgen, use_far, 0ull, 0ull};
            expand_small(a.index, qcur, nq, a.tasks, &ctl->tasks[cur], gwarp, nwarps, relax);
            unsigned long long mfb = block_sum(relax.mf, s_red);
            if (threadIdx.x == 0 && mfb) atomicAdd(&ctl->mf[nxt], mfb);
            relax.mf = 0;
            if (!grid_barrier(&ctl->gs)) return;
            const int nt = __ldcg(&ctl->tasks[cur]);
            if (nt > 0) {
                expand_tasks(a.index, a.tasks, nt, gwarp, nwarps, relax);
                mfb = block_sum(relax.mf, s_red);
                if (threadIdx.x == 0 && mfb) atomicAdd(&ctl->mf[nxt], mfb);
                if (!grid_barrier(&ctl->gs)) return;
            }
            if (kStats) my_e += relax.relaxed;
        }
        E++;
    }
    if (kStats) {
        unsigned long long v = block_sum(my_v, s_red);
        if (threadIdx.x == 0 && v) atomicAdd(&ctl->vproc, v);
        unsigned long long e = block_sum(my_e, s_red);
        if (threadIdx.x == 0 && e) atomicAdd(&ctl->erelax, e);
    }
    if (gtid == 0 && !__ldcg(&ctl->need_pull)) {
        ctl->finished = 1;
        ctl->epochs = E;
        ctl->phases = phase;
        ctl->pulls = pulls;
        ctl->trace[E < kTraceEpochs ? E : kTraceEpochs].t_ns = globaltimer_ns();
    }
}

// One pull epoch (the reference's Bellman-Ford epoch) as its own launch, so
// that it runs at the occupancy of a small kernel instead of the persistent
// kernel's; lowered rows are marked in `changed`.
template <bool kStats>
__global__ void __launch_bounds__(kPullThreads, 6) sssp_pull_kernel(SsspArgs a) {
    __shared__ int32_t s_acc[kPullThreads / 32][32];
    __shared__ unsigned long long s_red[32];
    // A speculative launch with no pull epoch pending returns at once.
    if (!__ldcg(&a.ctl->need_pull) || __ldcg(&a.ctl->gs.err)) return;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    // Every distance this sweep starts from reaches all its neighbours' rows
    // (a value that falls during the sweep marks its row changed), so the far
    // pile's entries need no later relaxation: drop them.  The resumed launch
    // re-queues the lowered rows under a new far claim.
    if (gtid == 0) a.ctl->far_len[__ldcg(&a.ctl->saved_phase) & 1] = 0;
    unsigned long long my_e = 0, my_mf = 0;
    pull_sweep<kStats>(a, gtid >> 5, (gridDim.x * blockDim.x) >> 5, s_acc, my_e, __ldcg(&a.ctl->saved_T), my_mf);
    const unsigned long long mf = block_sum(my_mf, s_red);
    if (threadIdx.x == 0 && mf) atomicAdd(&a.ctl->pull_mf, mf);
    if (kStats) {
        __syncthreads();
        const unsigned long long e = block_sum(my_e, s_red);
        if (threadIdx.x == 0 && e) atomicAdd(&a.ctl->erelax, e);
    }
}

// Shortest-path tree: any u with dist[u] + w(u->v) == dist[v] is a valid
// parent (weights are non-negative integers).  Warp per source row, push
// direction, so directed weights are read from the row that owns them.
__global__ void sssp_parent_init(int32_t *parent, int32_t n, int32_t src) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        parent[v] = v == src ? src : -1;
}

__global__ void sssp_parents_fill(const int64_t *index, const int32_t *nbr, const int32_t *w, const int32_t *dist,
                                  int32_t n, int32_t src, int32_t *parent) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += nw) {
        const int32_t du = dist[u];
        if (du == kInfDist) continue;
        const int64_t b = index[u], e = index[u + 1];
        for (int64_t i = b + lane; i < e; i += 32) {
            const int32_t v = nbr[i];
            if (v != src && sat_add(du, w[i]) == dist[v]) parent[v] = u;
        }
    }
}

__global__ void count_finite(const int32_t *dist, int32_t n, unsigned long long *out) {
    __shared__ unsigned long long s_red[32];
    unsigned long long c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        c += dist[i] != kInfDist;
    c = block_sum(c, s_red);
    if (threadIdx.x == 0 && c) atomicAdd(out, c);
}

// Candidates are clamped at INT32_MAX (sat_add).  When every finite
// distance plus the largest weight stays below the clamp, no candidate
// reached it, so the clamp changed nothing; otherwise some distance may lie
// beyond int32 and the run is refused.  Sets *flag when a finite distance
// exceeds `limit` (INT32_MAX - 1 - largest weight).
__global__ void any_above(const int32_t *dist, int32_t n, int32_t limit, int *flag) {
    bool hi = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t d = dist[i];
        hi |= d != kInfDist && d > limit;
    }
    if (__any_sync(kFull, hi) && (threadIdx.x & 31) == 0) *flag = 1;
}

// Whether any weight is negative (flags[0]), the largest weight (flags[1])
// and the weights' sum.
__global__ void weight_stats(const int64_t *index, const int32_t *w, int32_t n, int *flags, unsigned long long *sum) {
    __shared__ unsigned long long s_red[32];
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long s = 0;
    int32_t mx = 0;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const int64_t b = index[v], e = index[v + 1];
        for (int64_t i = b + lane; i < e; i += 32) {
            const int32_t x = w[i];
            if (x < 0) flags[0] = 1;
            s += (unsigned long long)max(x, 0);
            mx = max(mx, x);
        }
    }
    mx = __reduce_max_sync(kFull, mx);
    if (lane == 0 && mx > 0) atomicMax(flags + 1, mx);
    s = block_sum(s, s_red);
    if (threadIdx.x == 0 && s) atomicAdd(sum, s);
}

// The pull sweeps' pair array: each row's (neighbour, weight) pairs ordered
// by weight bucket, stable within a bucket (CSR order), so the result is the
// same on every run.  One warp per row: a bucket histogram in shared memory,
// its exclusive scan, then a stable scatter 32 pairs at a time (lanes of one
// bucket take consecutive slots in lane order).
constexpr int kOrderThreads = 256;
__global__ void __launch_bounds__(kOrderThreads) weight_order_rows(const int64_t *index, const int32_t *nbr,
                                                                   const int32_t *w, int32_t n, int ws,
                                                                   int2 *adj) {
    __shared__ int s_cnt[kOrderThreads / 32][256];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int *cnt = s_cnt[wib];
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const int64_t b = index[v], e = index[v + 1];
        if (e - b <= 1) {
            if (e > b && lane == 0) adj[b] = make_int2(nbr[b], w[b]);
            continue;
        }
#pragma unroll
        for (int k = 0; k < 8; k++) cnt[lane * 8 + k] = 0;
        __syncwarp();
        for (int64_t i = b + lane; i < e; i += 32) atomicAdd(&cnt[wbucket(w[i], ws)], 1);
        __syncwarp();
        int loc[8], tot = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            loc[k] = tot;
            tot += cnt[lane * 8 + k];
        }
        int incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 8; k++) cnt[lane * 8 + k] = incl - tot + loc[k];
        __syncwarp();
        for (int64_t i0 = b; i0 < e; i0 += 32) {
            const int64_t i = i0 + lane;
            const bool act = i < e;
            int2 q = make_int2(0, 0);
            int bk = -1;
            if (act) {
                q = make_int2(nbr[i], w[i]);
                bk = wbucket(q.y, ws);
            }
            const unsigned peers = __match_any_sync(kFull, bk);
            if (act) adj[b + cnt[bk] + __popc(peers & ((1u << lane) - 1u))] = q;
            __syncwarp();
            if (act && (peers >> lane) == 1u) cnt[bk] += __popc(peers);  // the bucket's highest lane
            __syncwarp();
        }
        __syncwarp();
    }
}

template <bool kStats>
hc_status launch_sssp(hc_graph *g, const SsspArgs &args) {
    static int blocks_per_sm[2] = {0, 0};
    int &bps = blocks_per_sm[kStats ? 1 : 0];
    if (bps == 0) {
        HC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, sssp_persistent<kStats>, kSsspThreads, 0));
        if (bps < 1) return fail(HC_ERR_CUDA, "SSSP kernel cannot be resident");
    }
    const int use = g->tune.sssp_blocks_per_sm > 0 ? std::min(bps, g->tune.sssp_blocks_per_sm) : bps;
    dim3 grid(g->sm_count * use), block(kSsspThreads);
    SsspArgs a = args;
    void *params[] = {&a};
    ::hc::count_launch();
    HC_CUDA_TRY(cudaLaunchCooperativeKernel((void *)sssp_persistent<kStats>, grid, block, params, 0, g->stream));
    return HC_OK;
}

template <bool kStats>
hc_status launch_pull(hc_graph *g, const SsspArgs &a) {
    static int blocks_per_sm[2] = {0, 0};
    int &bps = blocks_per_sm[kStats ? 1 : 0];
    if (bps == 0) {
        HC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, sssp_pull_kernel<kStats>, kPullThreads, 0));
        if (bps < 1) return fail(HC_ERR_CUDA, "SSSP pull kernel cannot be resident");
    }
    ::hc::count_launch();
    sssp_pull_kernel<kStats><<<g->sm_count * bps, kPullThreads, 0, g->stream>>>(a);
    HC_CUDA_TRY(cudaGetLastError());
    return HC_OK;
}

// One source: the persistent kernel, and for each pull epoch it hands back,
// the pull kernel and another persistent launch that resumes the loop.  The
// chain is queued kSpeculate (pull, resume) pairs at a time without waiting
// for the host: a pull launch with no epoch pending and a persistent launch
// after the end return at once.  The host checks once per batch.
constexpr int kSpeculate = 3;

template <bool kStats>
hc_status run_source(hc_graph *g, const SsspArgs &a) {
    HC_TRY(launch_sssp<kStats>(g, a));
    if (a.pull_alpha <= 0) return HC_OK;  // no pull epochs: one launch
    for (int round = 0;; round++) {
        for (int k = 0; k < kSpeculate; k++) {
            HC_TRY(launch_pull<kStats>(g, a));
            HC_TRY(launch_sssp<kStats>(g, a));
        }
        // gs.err, need_pull, resume and finished, at the head of SsspCtl.
        const void *h_head = nullptr;
        HC_TRY(ctl_read(g, a.ctl, offsetof(SsspCtl, finished) + sizeof(int), 3, &h_head));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        SsspCtl head;
        std::memcpy(&head, h_head, offsetof(SsspCtl, finished) + sizeof(int));
        if (head.gs.err || head.finished) return HC_OK;
        if ((int64_t)round * kSpeculate > a.max_epochs)
            return fail(HC_ERR_NOT_CONVERGED, "hc_sssp: pull rounds exceed the epoch cap");
    }
}

}  // namespace

// The bucket shift for weights in [0, w_max]: the smallest ws with w_max >> ws < 256.
int weight_shift(int32_t w_max) {
    int ws = 0;
    while ((w_max >> ws) > 255) ws++;
    return ws;
}

// Builds the pull sweeps' weight-ordered pair array once per graph (after the
// weight statistics, which give the bucket shift).
hc_status ensure_weight_order(hc_graph *g) {
    if (g->sssp_adj_ready) return HC_OK;
    HC_TRY(g->sssp_adj.ensure(sizeof(int2) * ((size_t)g->M + 64)));
    {
        weight_order_rows<<<g->sm_count * 8, kOrderThreads, 0, g->stream>>>(
            g->index.as<int64_t>(), g->nbr.as<int32_t>(), g->wgt.as<int32_t>(), g->N, weight_shift(g->w_max),
            g->sssp_adj.as<int2>());
        ::hc::count_launch();
    }
    HC_CUDA_TRY(cudaGetLastError());
    g->sssp_adj_ready = 1;
    return HC_OK;
}

hc_status ensure_weight_stats(hc_graph *g) {
    if (g->wstats_done) return HC_OK;
    DevBuf buf;
    HC_TRY(buf.ensure(64));
    HC_CUDA_TRY(cudaMemsetAsync(buf.ptr, 0, 64, g->stream));
    int *flags = buf.as<int>();
    unsigned long long *sum = reinterpret_cast<unsigned long long *>(buf.as<char>() + 16);
    {
        weight_stats<<<g->sm_count * 8, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->wgt.as<int32_t>(), g->N,
                                                             flags, sum);
        ::hc::count_launch();
    }
    HC_CUDA_TRY(cudaGetLastError());
    int hf[2] = {0, 0};
    unsigned long long hsum = 0;
    HC_CUDA_TRY(cudaMemcpyAsync(hf, flags, 8, cudaMemcpyDeviceToHost, g->stream));
    HC_CUDA_TRY(cudaMemcpyAsync(&hsum, sum, 8, cudaMemcpyDeviceToHost, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    g->w_negative = hf[0];
    g->w_max = hf[1];
    // Symmetric weights (w(u->v) == w(v->u) for every edge): one hashing pass.
    bool st = false, ws = false;
    HC_TRY(edge_symmetry(g, reinterpret_cast<const uint32_t *>(g->wgt.ptr), &st, &ws));
    g->w_symmetric = ws;
    g->w_mean = g->M ? (double)hsum / (double)g->M : 1.0;
    g->wstats_done = 1;
    return HC_OK;
}

}  // namespace hc

using namespace hc;

extern "C" hc_status hc_sssp(hc_graph *g, const int32_t *sources, int32_t num_sources, int32_t *dist_out,
                             int32_t *parent_out, const hc_sssp_opts *opts, hc_sssp_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    ReclaimScope reclaim_scope(g, kKeepAdj);
    if (!sources || num_sources < 0) return fail(HC_ERR_INVALID_ARG, "hc_sssp: bad source list");
    if (g->wtype != HC_W_I32) return fail(HC_ERR_UNSUPPORTED, "hc_sssp: graph needs int32 edge weights");
    hc_sssp_opts o{};
    if (opts) o = *opts;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    std::vector<int32_t> src(num_sources);
    HC_CUDA_TRY(cudaMemcpy(src.data(), sources, sizeof(int32_t) * num_sources, cudaMemcpyDefault));
    for (int32_t s : src)
        if (s < 0 || s >= g->N) return fail(HC_ERR_INVALID_ARG, "hc_sssp: source %d outside [0, %d)", s, g->N);

    // Weights must be non-negative; the mean weight sets the default delta.
    HC_TRY(ensure_weight_stats(g));
    if (g->w_negative) return fail(HC_ERR_INVALID_ARG, "hc_sssp: negative edge weight");
    HC_TRY(ensure_plan(g));

    const int64_t n = g->N;
    const int64_t W = (n + 31) / 32;
    const int64_t ntasks = max_expand_tasks(g->M, n);
    HC_TRY(g->ws_sssp.ensure(sizeof(int32_t) * 6 * n + 4 * W + sizeof(int2) * ntasks + 4096));
    HC_TRY(g->ws_ctl.ensure(4096));
    char *p = g->ws_sssp.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    SsspArgs a{};
    a.index = g->index.as<int64_t>();
    a.nbr = g->nbr.as<int32_t>();
    a.w = g->wgt.as<int32_t>();
    a.n = g->N;
    a.n_active = g->n_active;
    a.m = g->M;
    a.q0 = (int32_t *)take(4 * n);
    a.q1 = (int32_t *)take(4 * n);
    a.far0 = (int32_t *)take(4 * n);
    a.far1 = (int32_t *)take(4 * n);
    a.stamp = (int32_t *)take(4 * n);
    a.fstamp = (int32_t *)take(4 * n);
    a.changed = (uint32_t *)take(4 * W);
    a.tasks = (int2 *)take(sizeof(int2) * ntasks);
    a.ctl = g->ws_ctl.as<SsspCtl>();
    a.plan = g->pr_view;
    a.max_epochs = o.max_epochs > 0 ? o.max_epochs : 0x7fffffff;
    // The pull sweep reads w(u->v) from v's row: only valid when weights are symmetric.
    // Zero fields: the handle's tuned values, else the defaults.
    if (o.pull_alpha == 0) o.pull_alpha = g->tune.sssp_pull_alpha;
    if (o.delta == 0) o.delta = g->tune.sssp_delta;
    a.pull_alpha = !g->w_symmetric ? 0 : (o.pull_alpha == 0 ? kDefaultPullAlpha : std::max(o.pull_alpha, 0));
    if (a.pull_alpha > 0) {
        HC_TRY(ensure_weight_order(g));
        a.adj = g->sssp_adj.as<int2>();
        a.ws = weight_shift(g->w_max);
    }
    if (o.delta == 0) {
        const double davg = g->n_active ? (double)g->M / (double)g->n_active : 1.0;
        a.delta = (int32_t)std::max(1.0, std::min(1e9, g->w_mean * 32.0 / std::max(davg, 1.0)));
    } else {
        a.delta = o.delta;
    }

    const bool dev_dist = is_device_pointer(dist_out);
    const bool dev_parent = is_device_pointer(parent_out);
    if (!dist_out) HC_TRY(g->ws_out0.ensure(4 * n));
    // Host outputs: staged on the device and copied while the next source runs.
    const bool host_dist = dist_out && !dev_dist, host_parent = parent_out && !dev_parent;
    OutPipe pipe;
    if (host_dist || host_parent) HC_TRY(pipe.init(g, 2, 4 * n));

    // Candidates can reach the INT32_MAX clamp only when a path of
    // n_active - 1 edges of the largest weight can; then each source's
    // distances are checked after its run (a flag in the control block's
    // spare half).
    static_assert(sizeof(SsspCtl) <= 2048, "SsspCtl overlaps its spare slots");
    const bool check_range = (int64_t)g->w_max * std::max<int64_t>(g->n_active - 1, 0) >= (int64_t)kInfDist;
    const int32_t range_limit = kInfDist - 1 - g->w_max;
    int *range_flag = (int *)((char *)a.ctl + 2056);
    double total_ms = 0;
    for (int32_t i = 0; i < num_sources; i++) {
        a.src = src[i];
        int32_t *stage[2] = {nullptr, nullptr};
        if (host_dist || host_parent) HC_TRY(pipe.acquire(i, stage));
        a.dist = dev_dist ? dist_out + (size_t)i * n : host_dist ? stage[0] : g->ws_out0.as<int32_t>();
        HC_TRY(ctl_zero(g, a.ctl, sizeof(SsspCtl)));
        HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
        HC_TRY(o.collect_stats ? run_source<true>(g, a) : run_source<false>(g, a));
        HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
        if (parent_out) {
            int32_t *par = dev_parent ? parent_out + (size_t)i * n : stage[1];
            { sssp_parent_init<<<g->sm_count * 4, 256, 0, g->stream>>>(par, g->N, a.src); ::hc::count_launch(); }
            { sssp_parents_fill<<<g->sm_count * 8, 256, 0, g->stream>>>(a.index, a.nbr, a.w, a.dist, g->N, a.src, par); ::hc::count_launch(); }
            HC_CUDA_TRY(cudaGetLastError());
        }
        if (host_dist || host_parent) {
            void *dst[2] = {host_dist ? (void *)(dist_out + (size_t)i * n) : nullptr,
                            host_parent ? (void *)(parent_out + (size_t)i * n) : nullptr};
            HC_TRY(pipe.release(i, dst));
        }
        SsspCtl c;
        int out_of_range = 0;
        const void *h_range = nullptr, *h_ctl = nullptr, *h_cnt = nullptr;
        if (check_range) {
            HC_TRY(ctl_zero(g, range_flag, sizeof(int)));
            { any_above<<<g->sm_count * 4, 256, 0, g->stream>>>(a.dist, g->N, range_limit, range_flag); ::hc::count_launch(); }
            HC_TRY(ctl_read(g, range_flag, sizeof(int), 1, &h_range));
        }
        HC_TRY(ctl_read(g, a.ctl, sizeof(c), 0, &h_ctl));
        if (o.collect_stats && stats) {
            unsigned long long *cnt = (unsigned long long *)((char *)a.ctl + 2048);
            HC_TRY(ctl_zero(g, cnt, 8));
            { count_finite<<<g->sm_count * 4, 256, 0, g->stream>>>(a.dist, g->N, cnt); ::hc::count_launch(); }
            HC_TRY(ctl_read(g, cnt, 8, 2, &h_cnt));
        }
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        std::memcpy(&c, h_ctl, sizeof(c));
        if (h_range) std::memcpy(&out_of_range, h_range, sizeof(int));
        if (h_cnt) {
            unsigned long long reached = 0;
            std::memcpy(&reached, h_cnt, 8);
            stats->reached += (int32_t)reached;
        }
        if (c.gs.err) return fail((hc_status)c.gs.err, "hc_sssp: device run from source %d ended with status %d",
                                  src[i], c.gs.err);
        if (out_of_range)
            return fail(HC_ERR_UNSUPPORTED, "hc_sssp: a distance from source %d comes within the largest weight "
                        "(%d) of INT32_MAX: int32 distances cannot hold it", src[i], g->w_max);
        float ms = 0;
        HC_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
        total_ms += ms;
        if (stats) {
            stats->epochs = std::max(stats->epochs, c.epochs);
            stats->vertices_processed += (int64_t)c.vproc;
            stats->edges_relaxed += (int64_t)c.erelax;
        }
        if (std::getenv("HC_TRACE")) {
            const int ne = std::min(c.epochs, kTraceEpochs);
            std::fprintf(stderr, "[hc sssp] src %d: %d epochs (%d pull), %d phases, delta %d, %.1f us\n", src[i],
                         c.epochs, c.pulls, c.phases, a.delta, ms * 1e3);
            for (int e = 0; e < ne; e++) {
                const int ph = c.trace[e].phase;
                std::fprintf(stderr, "[hc sssp]   E%-4d %s phase %-4d nq=%-9d %8.1f us\n", e, ph < 0 ? "pull" : "push",
                             ph < 0 ? -1 - ph : ph, c.trace[e].nq, (c.trace[e + 1].t_ns - c.trace[e].t_ns) * 1e-3);
            }
        }
    }
    if (host_dist || host_parent) HC_TRY(pipe.finish());
    if (stats) {
        stats->ms = total_ms;
        // 16 B offsets per processed vertex, 8 B (neighbour + weight) per
        // relaxed edge, 4 B distance write per reached vertex.
        stats->bytes_model = 16.0 * (double)stats->vertices_processed + 8.0 * (double)stats->edges_relaxed +
                             4.0 * (double)stats->reached;
    }
    return HC_OK;
}
