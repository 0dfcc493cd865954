// Batched multi-source SSSP.
//
// The reference runs sources one after another (src/benchmarks/gpu_benchmark.cuh:577-586),
// each a full Bellman-Ford pull (src/kernels/gpu/sssp.cuh:42-100).  Here a group
// of sources shares every sweep: distances are vertex-major, dist[v][K], lane l
// of a warp owns the SPL distance words l*SPL .. l*SPL+SPL-1 of a row and reads
// them with one SPL-wide vector load, so the distances of a vertex for the
// whole group are one contiguous row.  A word holds one int32 distance (wide)
// or two uint16 distances (narrow, see NarrowDist), so K = 32 * SPL or 64 * SPL
// sources.  An activity mask per vertex (bit l = one of lane l's distances
// dropped last epoch) and a queue of active vertices drive the epochs: every
// edge out of the queue is relaxed for the active lanes, a warp keeping four
// edges in flight (row loads, then atomic minimums, then the activity updates
// of the four targets).  Rows longer than kLongRow are cut into chunks
// processed by a second launch.  While the queue covers a large part of the
// graph (and weights are symmetric) an epoch is a pull instead: a warp per row
// takes the minimum over its active neighbours and writes the row once, so
// the hub rows that most edges point at are read, not hammered with atomics.
// Wider groups amortise the row reads over more sources; the frontiers of
// Kronecker sources overlap, so the union frontier grows more slowly than the
// group.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr int kLongRow = 2048;
// An epoch is a pull when the edges out of its queue, times kPullAlpha, exceed
// M: a pull reads every row of the distance matrix once, a push only the rows
// its queue's edges reach.
constexpr int kPullAlpha = 2;

// Distance words.
//
// Wide: one int32 distance per word, kInfDist unreachable.
//
// Narrow: two uint16 distances per word (source 2j of a lane's range in the
// low half of its word j), kInf16 unreachable, on graphs whose largest weight
// is at most kMsspNarrowMaxW.  A stored value is at most kInf16, so a value
// plus a weight stays below 0x10000 and the per-halfword add never wraps; a
// candidate at or above kInf16 never lowers anything, so a distance that does
// not fit stays unreachable instead of being wrong.  The group's distances are
// exact when the largest final finite distance plus the largest weight is
// below kInf16: every edge out of a reached vertex was then relaxed with that
// vertex's final value inside the range, so the result is the true fixed
// point.  The transpose that writes the output checks this, and a group that
// fails the check runs again with wide words.  The kernels also keep the
// largest finite value they write (every final value is one of them), and the
// epoch loop stops early once that plus the largest weight reaches kInf16, so
// a graph of long distances costs a few epochs, not a full run.  Half the
// bytes per row read, and one add-min instruction per two distances.
constexpr uint32_t kInf16 = 0xF000u;
// MsspCtl.status of a narrow group stopped because its distances may not fit.
constexpr int kStatusRange = 0x7FFF0001;

struct WideDist {
    using W = int32_t;
    static constexpr int kPer = 1;
    static constexpr W kInfWord = kInfDist;
    __device__ static W weight(int32_t w) { return w; }
    // d + w clamped at INT32_MAX: for d, w in [0, INT32_MAX] the unsigned
    // sum cannot wrap, and a clamped candidate lowers nothing (the transpose
    // refuses a group whose distances come within w_max of the clamp).
    __device__ static W sum(W d, W w) {
        const uint32_t s = (uint32_t)d + (uint32_t)w;
        return s < (uint32_t)kInfDist ? (W)s : kInfDist;
    }
    // min(best, d + w) over the word's distances; an unreachable d changes nothing.
    __device__ static W relax(W best, W d, W w) { return min(best, sum(d, w)); }
    // Push candidate d + w (unreachable stays unreachable).
    __device__ static W cand(W du, W w) { return sum(du, w); }
    __device__ static bool lowers(W nd, W d) { return nd < d; }
    __device__ static void atomic_lower(W *p, W nd, W) { atomicMin(p, nd); }
    __device__ static W lower_of(W a, W b) { return min(a, b); }
    __device__ static void note(W &, W) {}
};

struct NarrowDist {
    using W = uint32_t;
    static constexpr int kPer = 2;
    static constexpr W kInfWord = kInf16 | (kInf16 << 16);
    __device__ static W weight(int32_t w) { return (uint32_t)w * 0x00010001u; }
    __device__ static W relax(W best, W d, W w) { return __viaddmin_u16x2(d, w, best); }
    __device__ static W cand(W du, W w) { return __vadd2(du, w); }
    __device__ static bool lowers(W nd, W d) { return __vcmpltu2(nd, d) != 0u; }
    // Per-halfword minimum by compare-and-swap, starting from the value seen.
    // A failed swap means the word fell meanwhile (each halfword can fall at
    // most kInf16 times), so the loop ends well before its cap.
    __device__ static void atomic_lower(W *p, W nd, W seen) {
        W old = seen;
        for (int i = 0; i < 4 * (int)kInf16; i++) {
            const W nw = __vminu2(old, nd);
            if (nw == old) return;
            const W prev = atomicCAS(p, old, nw);
            if (prev == old) return;
            old = prev;
        }
    }
    __device__ static W lower_of(W a, W b) { return __vminu2(a, b); }
    // Running per-halfword maximum of the finite values written.
    __device__ static void note(W &mx, W x) { mx = __vmaxu2(mx, x & __vcmpltu2(x, kInfWord)); }
};

// Epoch control in device memory.  Every kernel of an epoch reads the queue
// length and the push/pull choice from here, so the same launch sequence runs
// from the host loop and as the body of a graph's while node, whose condition
// mssp_end sets.
struct MsspCtl {
    int qlen[2];                    // queue lengths; parity c reads qlen[c], fills qlen[c ^ 1]
    unsigned long long qedges[2];   // edges out of the vertices of each queue
    int ntasks;                     // long-row chunks queued by the push epoch
    int epochs;
    int stop;                       // the loop ended early (status says why)
    int status;
    int pull_alpha;                 // 0: push only
    int max_epochs;
    long long m;
    unsigned long long t0;
    unsigned maxf;                  // largest finite distance of the group (transpose)
    unsigned maxw;                  // largest finite distance written so far (narrow epochs)
    int w_max;                      // largest edge weight
    int narrow;                     // 16-bit distance words
};

__device__ __forceinline__ int ctl_queue(const MsspCtl *ctl, int c) { return ctl->stop ? 0 : ctl->qlen[c]; }
__device__ __forceinline__ bool ctl_pull(const MsspCtl *ctl, int c) {
    return ctl->pull_alpha > 0 && (double)ctl->qedges[c] * ctl->pull_alpha > (double)ctl->m;
}

// Folds a thread's running maximum of written halfwords into ctl->maxw (one
// atomic per warp; every lane of the warp calls it).
template <class D>
__device__ __forceinline__ void note_flush(MsspCtl *ctl, typename D::W mx) {
    if constexpr (D::kPer == 2) {
        unsigned m = max(mx & 0xFFFFu, mx >> 16);
        m = __reduce_max_sync(kFull, m);
        if ((threadIdx.x & 31) == 0 && m) atomicMax(&ctl->maxw, m);
    }
}

// A lane's SPL distance words of one vertex.  kL1: through L1 (neighbour
// rows, which many warps of an SM read: most edges point at a few thousand hub
// rows); a value cached earlier in the same launch may be stale, but
// distances only fall, so it is an upper bound, and the vertex that lowered
// it is active for the next epoch.  Otherwise L2 only (rows this warp owns).
template <int SPL, bool kL1 = false>
__device__ __forceinline__ void load_row(const int32_t *p, int32_t (&d)[SPL]) {
    if constexpr (SPL == 1) {
        d[0] = kL1 ? __ldca(p) : __ldcg(p);
    } else if constexpr (SPL == 2) {
        const int2 *q = reinterpret_cast<const int2 *>(p);
        const int2 x = kL1 ? __ldca(q) : __ldcg(q);
        d[0] = x.x;
        d[1] = x.y;
    } else {
#pragma unroll
        for (int h = 0; h < SPL / 4; h++) {
            const int4 *q = reinterpret_cast<const int4 *>(p) + h;
            const int4 x = kL1 ? __ldca(q) : __ldcg(q);
            d[4 * h] = x.x;
            d[4 * h + 1] = x.y;
            d[4 * h + 2] = x.z;
            d[4 * h + 3] = x.w;
        }
    }
}

template <int SPL, bool kL1 = false, class W>
__device__ __forceinline__ void load_words(const W *p, W (&d)[SPL]) {
    int32_t t[SPL];
    load_row<SPL, kL1>(reinterpret_cast<const int32_t *>(p), t);
#pragma unroll
    for (int s = 0; s < SPL; s++) d[s] = (W)t[s];
}

template <class D, int SPL>
__global__ void mssp_init(int32_t n, typename D::W *dist, uint32_t *act0, uint32_t *act1) {
    const size_t total = (size_t)n * 32 * SPL;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        dist[i] = D::kInfWord;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        act0[i] = 0;
        act1[i] = 0;
    }
}

// Source s of the group sits at distance slot s of each row (a halfword for
// narrow words) and belongs to lane s / (SPL * kPer).
template <class D, int SPL>
__global__ void mssp_seed(int nsrc, const int32_t *src, const int64_t *index, typename D::W *dist, uint32_t *act,
                          int32_t *queue, MsspCtl *ctl, int pull_alpha, long long m, int max_epochs, int w_max) {
    constexpr int K = 32 * SPL * D::kPer;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int q = 0;
        unsigned long long qe = 0;
        for (int s = 0; s < nsrc; s++) {
            const int32_t v = src[s];
            if constexpr (D::kPer == 1) {
                dist[(size_t)v * K + s] = 0;
            } else {
                reinterpret_cast<uint16_t *>(dist)[(size_t)v * K + s] = 0;
            }
            if (act[v] == 0) {
                queue[q++] = v;
                qe += (unsigned long long)(index[v + 1] - index[v]);
            }
            act[v] |= 1u << (s / (SPL * D::kPer));
        }
        MsspCtl c{};
        c.qlen[0] = q;
        c.qedges[0] = qe;
        c.pull_alpha = pull_alpha;
        c.m = m;
        c.max_epochs = max_epochs;
        c.w_max = w_max;
        c.narrow = D::kPer == 2;
        c.t0 = globaltimer_ns();
        *ctl = c;
    }
}

// Edges (push) or neighbours (pull) a warp keeps in flight: four, or two
// when a lane holds 16 words per vertex (register budget).
template <int SPL>
constexpr int kInflight = SPL >= 16 ? 2 : 4;

// Relax edges [e0, e1) of row u for the active lanes in `m`; du = this lane's
// distance words of u.
template <class D, int SPL>
__device__ __forceinline__ void relax_range(const int64_t *index, const int32_t *nbr, const int32_t *w,
                                            typename D::W *dist, uint32_t m, const typename D::W (&du)[SPL],
                                            int64_t e0, int64_t e1, uint32_t *act_next, int32_t *qnext, int *qlen,
                                            unsigned long long &relaxed, unsigned long long &qe,
                                            typename D::W &wmax) {
    using W = typename D::W;
    constexpr int KW = 32 * SPL;
    const int lane = threadIdx.x & 31;
    const bool on = (m >> lane) & 1u;
    for (int64_t base = e0; base < e1; base += 32) {
        const int64_t my = base + lane;
        const int cnt = (int)((e1 - base) < 32 ? (e1 - base) : 32);
        int32_t vv = 0, ww = 0;
        if (my < e1) {
            vv = nbr[my];
            ww = w[my];
        }
        constexpr int F = kInflight<SPL>;
        for (int j0 = 0; j0 < cnt; j0 += F) {
            int32_t v[F];
            W wt[F], d[F][SPL];
            bool ok[F], imp[F];
#pragma unroll
            for (int k = 0; k < F; k++) {
                const int idx = j0 + k;
                v[k] = __shfl_sync(kFull, vv, idx & 31);
                wt[k] = D::weight(__shfl_sync(kFull, ww, idx & 31));
                ok[k] = on && idx < cnt;
            }
#pragma unroll
            for (int k = 0; k < F; k++) {
                if (ok[k]) {
                    load_words<SPL, true>(dist + (size_t)v[k] * KW + lane * SPL, d[k]);
                } else {
#pragma unroll
                    for (int s = 0; s < SPL; s++) d[k][s] = D::kInfWord;
                }
            }
            // The update is a fire-and-forget atomic minimum; the target is
            // marked active whenever the loaded value was larger, which covers
            // every real improvement (values only fall between the load and
            // the atomic) at the price of an occasional redundant rescan.
#pragma unroll
            for (int k = 0; k < F; k++) {
                imp[k] = false;
#pragma unroll
                for (int s = 0; s < SPL; s++) {
                    const W nd = D::cand(du[s], wt[k]);
                    if (ok[k] && D::lowers(nd, d[k][s])) {
                        D::atomic_lower(dist + (size_t)v[k] * KW + lane * SPL + s, nd, d[k][s]);
                        D::note(wmax, D::lower_of(nd, d[k][s]));  // only the halves that fell
                        imp[k] = true;
                    }
                }
            }
            unsigned mybal = 0u;  // lane k < F: target k's new activity bits
            int32_t myv = 0;
#pragma unroll
            for (int k = 0; k < F; k++) {
                const unsigned b = __ballot_sync(kFull, imp[k]);
                if (lane == k) {
                    mybal = b;
                    myv = v[k];
                }
            }
            bool app = false;
            if (mybal) app = atomicOr(act_next + myv, mybal) == 0u;
            const unsigned ap = __ballot_sync(kFull, app);
            if (ap) {
                int base_q = 0;
                const int leader = __ffs(ap) - 1;
                if (lane == leader) base_q = atomicAdd(qlen, __popc(ap));
                base_q = __shfl_sync(kFull, base_q, leader);
                if (app) {
                    qnext[base_q + __popc(ap & ((1u << lane) - 1u))] = myv;
                    qe += (unsigned long long)(index[myv + 1] - index[myv]);
                }
            }
        }
        if (lane == 0) relaxed += (unsigned long long)cnt * __popc(m) * SPL * D::kPer;
    }
}

template <class D, int SPL>
__global__ void __launch_bounds__(256) mssp_epoch(const int64_t *index, const int32_t *nbr, const int32_t *w,
                                                  typename D::W *dist, const int32_t *qcur, const uint32_t *act_cur,
                                                  uint32_t *act_next, int32_t *qnext, int2 *tasks, MsspCtl *ctl, int c,
                                                  unsigned long long *relaxed) {
    const int nq = ctl_queue(ctl, c);
    if (nq == 0 || ctl_pull(ctl, c)) return;
    int *qnext_len = &ctl->qlen[c ^ 1];
    int *ntasks = &ctl->ntasks;
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long rel = 0, qe = 0;
    typename D::W wmax = 0;
    for (int qi = gwarp; qi < nq; qi += nwarps) {
        const int32_t u = qcur[qi];
        const uint32_t m = act_cur[u];
        const int64_t b = index[u], e = index[u + 1];
        if (e - b > kLongRow) {
            if (lane == 0) {
                const int nc = (int)((e - b + kLongRow - 1) / kLongRow);
                const int t0 = atomicAdd(ntasks, nc);
                for (int c = 0; c < nc; c++) tasks[t0 + c] = make_int2(u, c);
            }
            continue;
        }
        typename D::W du[SPL];
        load_words<SPL>(dist + (size_t)u * 32 * SPL + lane * SPL, du);
        relax_range<D, SPL>(index, nbr, w, dist, m, du, b, e, act_next, qnext, qnext_len, rel, qe, wmax);
    }
    note_flush<D>(ctl, wmax);
    rel = warp_sum(rel);
    qe = warp_sum(qe);
    if (lane == 0 && rel) atomicAdd(relaxed, rel);
    if (lane == 0 && qe) atomicAdd(&ctl->qedges[c ^ 1], qe);
}

template <class D, int SPL>
__global__ void __launch_bounds__(256) mssp_tasks(const int64_t *index, const int32_t *nbr, const int32_t *w,
                                                  typename D::W *dist, const int2 *tasks, const uint32_t *act_cur,
                                                  uint32_t *act_next, int32_t *qnext, MsspCtl *ctl, int c,
                                                  unsigned long long *relaxed) {
    const int nq = ctl_queue(ctl, c);
    if (nq == 0 || ctl_pull(ctl, c)) return;
    int *qnext_len = &ctl->qlen[c ^ 1];
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nt = ctl->ntasks;
    unsigned long long rel = 0, qe = 0;
    typename D::W wmax = 0;
    for (int t = gwarp; t < nt; t += nwarps) {
        const int2 tk = tasks[t];
        const int32_t u = tk.x;
        const uint32_t m = act_cur[u];
        const int64_t rb = index[u], re = index[u + 1];
        const int64_t b = rb + (int64_t)tk.y * kLongRow;
        const int64_t e = (re < b + kLongRow) ? re : b + kLongRow;
        typename D::W du[SPL];
        load_words<SPL>(dist + (size_t)u * 32 * SPL + lane * SPL, du);
        relax_range<D, SPL>(index, nbr, w, dist, m, du, b, e, act_next, qnext, qnext_len, rel, qe, wmax);
    }
    note_flush<D>(ctl, wmax);
    rel = warp_sum(rel);
    qe = warp_sum(qe);
    if (lane == 0 && rel) atomicAdd(relaxed, rel);
    if (lane == 0 && qe) atomicAdd(&ctl->qedges[c ^ 1], qe);
}

// Pull epoch, used while the queue covers a large part of the graph (weights
// symmetric, so w(u->v) is read from v's row).  Items [row_begin, row_end)
// are rows of at most kLongRow edges, one warp each, the only writer of that
// row; the items after them are kLongRow-edge chunks of the longer rows, which
// merge with atomic minimums.  A warp takes the minimum over the neighbours
// whose activity mask has its lane's bit, four neighbours in flight, and
// writes the row and its activity mask once.
//
// An epoch runs in two launches on degree-sorted graphs: the hub prefix (the
// rows holding half the edges, and the long-row chunks) first, then the other
// rows, which count a neighbour as active when it changed in the previous
// epoch or in this one (`fresh`): most shortest paths pass through hubs, so an
// improvement travels two hops per epoch.  Any order of pulls is valid, since
// distances only fall and a lowered row is active for the next epoch.
template <class D, int SPL>
__global__ void __launch_bounds__(256) mssp_pull(const int64_t *index, const int32_t *nbr, const int32_t *w,
                                                 typename D::W *dist, int32_t row_begin, int32_t row_end,
                                                 const int2 *tasks, int ntasks, const uint32_t *act_cur,
                                                 uint32_t *act_next, int fresh, MsspCtl *ctl, int c,
                                                 unsigned long long *relaxed) {
    using W = typename D::W;
    const int nq = ctl_queue(ctl, c);
    if (nq == 0 || !ctl_pull(ctl, c)) return;
    constexpr int KW = 32 * SPL;
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long rel = 0;
    W wmax = 0;
    const int32_t n_rows = row_end - row_begin;
    const int64_t total = (int64_t)n_rows + ntasks;
    for (int64_t it = gwarp; it < total; it += nwarps) {
        int32_t v;
        int64_t b, e;
        bool chunk;
        if (it < n_rows) {
            v = row_begin + (int32_t)it;
            b = index[v];
            e = index[v + 1];
            if (e == b || e - b > kLongRow) continue;
            chunk = false;
        } else {
            const int2 tk = tasks[it - n_rows];
            v = tk.x;
            const int64_t re = index[v + 1];
            b = index[v] + (int64_t)tk.y * kLongRow;
            e = (re < b + kLongRow) ? re : b + kLongRow;
            chunk = true;
        }
        W *row = dist + (size_t)v * KW + lane * SPL;
        W dv[SPL], best[SPL];
        load_words<SPL>(row, dv);
#pragma unroll
        for (int s = 0; s < SPL; s++) best[s] = dv[s];
        for (int64_t base = b; base < e; base += 32) {
            const int64_t my = base + lane;
            int32_t uu = 0, ww = 0;
            uint32_t aa = 0;
            if (my < e) {
                uu = nbr[my];
                ww = w[my];
                aa = __ldcg(act_cur + uu);
                // A hub row (below row_begin) may have changed earlier in this epoch.
                if (fresh && uu < row_begin) aa |= __ldcg(act_next + uu);
            }
            rel += (unsigned long long)__popc(aa) * SPL * D::kPer;
            unsigned live = __ballot_sync(kFull, aa != 0u);
            while (live) {
                constexpr int F = kInflight<SPL>;
                int32_t u[F];
                W wt[F], d[F][SPL];
                bool on[F];
#pragma unroll
                for (int k = 0; k < F; k++) {
                    const bool have = live != 0u;
                    const int idx = have ? __ffs(live) - 1 : 0;
                    if (have) live &= live - 1u;
                    u[k] = __shfl_sync(kFull, uu, idx);
                    wt[k] = D::weight(__shfl_sync(kFull, ww, idx));
                    const uint32_t a = __shfl_sync(kFull, aa, idx);
                    on[k] = have && ((a >> lane) & 1u);
                }
#pragma unroll
                for (int k = 0; k < F; k++) {
                    if (on[k]) {
                        load_words<SPL, true>(dist + (size_t)u[k] * KW + lane * SPL, d[k]);
                    } else {
#pragma unroll
                        for (int s = 0; s < SPL; s++) d[k][s] = D::kInfWord;
                    }
                }
#pragma unroll
                for (int k = 0; k < F; k++) {
#pragma unroll
                    for (int s = 0; s < SPL; s++) best[s] = D::relax(best[s], d[k][s], wt[k]);
                }
            }
        }
        // best <= dv slot by slot, so any difference is an improvement.
        bool imp = false;
#pragma unroll
        for (int s = 0; s < SPL; s++) imp |= best[s] != dv[s];
        const unsigned bal = __ballot_sync(kFull, imp);
        if (!bal) continue;
#pragma unroll
        for (int s = 0; s < SPL; s++) D::note(wmax, best[s]);
        if (chunk) {
#pragma unroll
            for (int s = 0; s < SPL; s++)
                if (best[s] != dv[s]) D::atomic_lower(row + s, best[s], dv[s]);
            if (lane == 0) atomicOr(act_next + v, bal);
        } else {
            if (imp) {
#pragma unroll
                for (int s = 0; s < SPL; s++) row[s] = best[s];
            }
            if (lane == 0) act_next[v] = bal;
        }
    }
    note_flush<D>(ctl, wmax);
    rel = warp_sum(rel);
    if (lane == 0 && rel) atomicAdd(relaxed, rel);
}

// Queue of the vertices with a non-zero activity mask, in vertex order (after
// a pull epoch).
__global__ void mssp_compact(const int64_t *index, const uint32_t *act, int32_t n, int32_t *q, MsspCtl *ctl, int c) {
    const int nq = ctl_queue(ctl, c);
    if (nq == 0 || !ctl_pull(ctl, c)) return;
    int *qlen = &ctl->qlen[c ^ 1];
    unsigned long long qe = 0;
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = gwarp * 32; base < n; base += nwarps * 32) {
        const int64_t v = base + lane;
        const bool on = v < n && act[v] != 0u;
        const unsigned bal = __ballot_sync(kFull, on);
        if (!bal) continue;
        int q0 = 0;
        if (lane == 0) q0 = atomicAdd(qlen, __popc(bal));
        q0 = __shfl_sync(kFull, q0, 0);
        if (on) {
            q[q0 + __popc(bal & ((1u << lane) - 1u))] = (int32_t)v;
            qe += (unsigned long long)(index[v + 1] - index[v]);
        }
    }
    qe = warp_sum(qe);
    if (lane == 0 && qe) atomicAdd(&ctl->qedges[c ^ 1], qe);
}

// (row, chunk) tasks for the rows longer than kLongRow.
__global__ void mssp_plan(const int64_t *index, int32_t n, int2 *tasks, int *ntasks) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t deg = index[v + 1] - index[v];
        if (deg <= kLongRow) continue;
        const int nc = (int)((deg + kLongRow - 1) / kLongRow);
        const int t0 = atomicAdd(ntasks, nc);
        for (int c = 0; c < nc; c++) tasks[t0 + c] = make_int2((int32_t)v, c);
    }
}

hc_status ensure_pull_plan(hc_graph *g) {
    if (g->mssp_tasks >= 0) return HC_OK;
    const int64_t max_tasks = 2 * (g->M / kLongRow) + 1;
    HC_TRY(g->ws_plan_mssp.ensure(sizeof(int2) * max_tasks + 256));
    int *cnt = reinterpret_cast<int *>(g->ws_plan_mssp.as<char>() + sizeof(int2) * max_tasks);
    HC_CUDA_TRY(cudaMemsetAsync(cnt, 0, 4, g->stream));
    { mssp_plan<<<g->sm_count * 8, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->N, g->ws_plan_mssp.as<int2>(), cnt); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    int h = 0;
    HC_CUDA_TRY(cudaMemcpyAsync(&h, cnt, 4, cudaMemcpyDeviceToHost, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    g->mssp_tasks = h;
    // Hub prefix of a degree-sorted graph: the fewest rows holding half the
    // edges (binary search over the offsets, a few 8-byte reads).
    g->mssp_hub_rows = g->n_active;
    if (g->degree_sorted && g->n_active > 0) {
        int32_t lo = 0, hi = g->n_active;
        while (lo < hi) {
            const int32_t mid = lo + (hi - lo) / 2;
            int64_t off = 0;
            HC_CUDA_TRY(cudaMemcpy(&off, g->index.as<int64_t>() + mid, sizeof(off), cudaMemcpyDeviceToHost));
            if (off >= g->M / 2) hi = mid; else lo = mid + 1;
        }
        g->mssp_hub_rows = std::max<int32_t>(lo, 1);
    }
    return HC_OK;
}

// Clears the activity masks of the epoch's queue (they become the next-next
// epoch's output).
__global__ void mssp_clear(const int32_t *q, uint32_t *act, const MsspCtl *ctl, int c) {
    const int nq = ctl_queue(ctl, c);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) act[q[i]] = 0;
}

// Closes epoch parity c: counts it, resets its counters for reuse, and decides
// whether another epoch runs (queue non-empty, under the epoch cap and the
// time bound, and for narrow words inside the 16-bit range); inside a graph
// it sets the while node's condition.
__global__ void mssp_end(MsspCtl *ctl, int c, cudaGraphConditionalHandle cond, int use_cond) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    bool go = false;
    if (!ctl->stop && ctl->qlen[c] > 0) {
        ctl->epochs++;
        ctl->qlen[c] = 0;
        ctl->qedges[c] = 0;
        ctl->ntasks = 0;
        go = ctl->qlen[c ^ 1] > 0;
        if (go && ctl->epochs >= ctl->max_epochs) {
            ctl->stop = 1;
            ctl->status = HC_ERR_NOT_CONVERGED;
            go = false;
        }
        if (go && globaltimer_ns() - ctl->t0 > c_limits.loop_ns) {
            ctl->stop = 1;
            ctl->status = HC_ERR_TIMEOUT;
            go = false;
        }
        if (ctl->narrow && (long long)ctl->maxw + ctl->w_max >= (long long)kInf16) {
            ctl->stop = 1;
            ctl->status = kStatusRange;
            go = false;
        }
    }
    if (use_cond) cudaGraphSetConditional(cond, go ? 1u : 0u);
}

// dist[v][K] -> out[s][v] (int32, unreachable = kInfDist) for the group's
// sources, vertex tiles through shared memory (coalesced reads of rows,
// coalesced writes per source).  Narrow words also yield the largest finite
// distance (ctl->maxf); out may then be null (the check alone).
template <class D, int SPL>
__global__ void mssp_transpose(const typename D::W *dist, int32_t n, int nsrc, int32_t *out, MsspCtl *ctl) {
    constexpr int KW = 32 * SPL;
    constexpr int K = KW * D::kPer;
    constexpr int TV = K >= 1024 ? 8 : K >= 512 ? 16 : 32;  // vertices per tile (<= 33 KB of shared memory)
    __shared__ int32_t tile[TV][K + 1];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    unsigned mx = 0;
    for (int64_t vb = (int64_t)blockIdx.x * TV; vb < n; vb += (int64_t)gridDim.x * TV) {
        for (int r = ty; r < TV; r += 8) {
            const int64_t v = vb + r;
            for (int c = tx; c < KW; c += 32) {
                const typename D::W x = v < n ? dist[(size_t)v * KW + c] : D::kInfWord;
                if constexpr (D::kPer == 1) {
                    if (x != kInfDist) mx = max(mx, (unsigned)x);
                    tile[r][c] = x;
                } else {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const unsigned hv = (x >> (16 * h)) & 0xFFFFu;
                        const bool fin = hv < kInf16;
                        if (fin) mx = max(mx, hv);
                        tile[r][2 * c + h] = fin ? (int32_t)hv : kInfDist;
                    }
                }
            }
        }
        __syncthreads();
        if (out) {
            for (int s = ty; s < nsrc; s += 8) {
                const int64_t v = vb + tx;
                if (tx < TV && v < n) out[(size_t)s * n + v] = tile[tx][s];
            }
        }
        __syncthreads();
    }
    mx = __reduce_max_sync(kFull, mx);
    if (tx == 0 && mx) atomicMax(&ctl->maxf, mx);
}

template <class D>
struct MsspBufs {
    typename D::W *dist;
    uint32_t *act[2];
    int32_t *q[2];
    int2 *tasks;
    MsspCtl *ctl;
    int32_t *src;
};

// One epoch of parity c: the push kernels, the pull kernels (each returns at
// once when the epoch is of the other kind), the activity clear and the end
// kernel.
template <class D, int SPL>
void launch_epoch(const hc_graph *g, cudaStream_t st, const MsspBufs<D> &b, int c, unsigned long long *relaxed,
                  cudaGraphConditionalHandle cond, int use_cond) {
    const int grid = g->sm_count * 8;
    const int64_t *index = g->index.as<int64_t>();
    const int32_t *nbr = g->nbr.as<int32_t>(), *w = g->wgt.as<int32_t>();
    mssp_epoch<D, SPL><<<grid, 256, 0, st>>>(index, nbr, w, b.dist, b.q[c], b.act[c], b.act[c ^ 1], b.q[c ^ 1],
                                             b.tasks, b.ctl, c, relaxed);
    mssp_tasks<D, SPL><<<grid, 256, 0, st>>>(index, nbr, w, b.dist, b.tasks, b.act[c], b.act[c ^ 1], b.q[c ^ 1],
                                             b.ctl, c, relaxed);
    const int32_t hub = g->mssp_hub_rows > 0 ? g->mssp_hub_rows : g->n_active;
    mssp_pull<D, SPL><<<grid, 256, 0, st>>>(index, nbr, w, b.dist, 0, hub, g->ws_plan_mssp.as<int2>(),
                                            g->mssp_tasks < 0 ? 0 : g->mssp_tasks, b.act[c], b.act[c ^ 1], 0, b.ctl,
                                            c, relaxed);
    if (hub < g->n_active)
        mssp_pull<D, SPL><<<grid, 256, 0, st>>>(index, nbr, w, b.dist, hub, g->n_active, nullptr, 0, b.act[c],
                                                b.act[c ^ 1], 1, b.ctl, c, relaxed);
    mssp_clear<<<grid, 256, 0, st>>>(b.q[c], b.act[c], b.ctl, c);
    mssp_compact<<<grid, 256, 0, st>>>(index, b.act[c ^ 1], g->N, b.q[c ^ 1], b.ctl, c);
    mssp_end<<<1, 32, 0, st>>>(b.ctl, c, cond, use_cond);
}
constexpr int kEpochLaunches = 7;

// One group of k <= 32 * SPL * kPer sources.  For narrow words *fits is set
// false when the distances may not all fit (the caller reruns the group wide);
// dst then holds no valid result.
template <class D, int SPL>
hc_status run_group(hc_graph *g, const int32_t *h_src, int k, int32_t *dst, int max_epochs, int pull_alpha,
                    bool use_graph, WhileGraph &eg, int *epochs_out, unsigned long long *relaxed, bool *fits) {
    using W = typename D::W;
    constexpr int KW = 32 * SPL;
    constexpr int K = KW * D::kPer;
    const int64_t n = g->N;
    const int64_t max_tasks = 2 * (g->M / kLongRow) + n / kLongRow + 64;
    HC_TRY(g->ws_batch.ensure((size_t)n * KW * 4 + (size_t)n * 4 * 4 + sizeof(int2) * max_tasks + 8192));
    char *p = g->ws_batch.as<char>();
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) / 256 * 256;
        return r;
    };
    MsspBufs<D> b;
    b.dist = (W *)take((size_t)n * KW * 4);
    b.act[0] = (uint32_t *)take((size_t)n * 4);
    b.act[1] = (uint32_t *)take((size_t)n * 4);
    b.q[0] = (int32_t *)take((size_t)n * 4);
    b.q[1] = (int32_t *)take((size_t)n * 4);
    b.tasks = (int2 *)take(sizeof(int2) * max_tasks);
    b.ctl = (MsspCtl *)take(sizeof(MsspCtl));
    b.src = (int32_t *)take(sizeof(int32_t) * K);
    const int grid = g->sm_count * 8;
    HC_TRY(g->pinned.ensure(2 * sizeof(MsspCtl) + 64));
    MsspCtl *hctl = g->pinned.as<MsspCtl>();
    HC_CUDA_TRY(cudaMemcpyAsync(b.src, h_src, sizeof(int32_t) * k, cudaMemcpyHostToDevice, g->stream));
    { mssp_init<D, SPL><<<grid, 256, 0, g->stream>>>(g->N, b.dist, b.act[0], b.act[1]); ::hc::count_launch(); }
    {
        mssp_seed<D, SPL><<<1, 32, 0, g->stream>>>(k, b.src, g->index.as<int64_t>(), b.dist, b.act[0], b.q[0], b.ctl,
                                                   pull_alpha, (long long)g->M, max_epochs, g->w_max);
        ::hc::count_launch();
    }
    HC_CUDA_TRY(cudaGetLastError());
    const bool trace = std::getenv("HC_TRACE") != nullptr;
    if (use_graph && !trace) {
        // The graph's body is two epochs (parity 0 then 1); kernels of an
        // epoch whose queue is empty return at once.
        if (!eg.exec) {
            auto body = [&](cudaStream_t cs, cudaGraphConditionalHandle cond) {
                launch_epoch<D, SPL>(g, cs, b, 0, relaxed, cond, 1);
                launch_epoch<D, SPL>(g, cs, b, 1, relaxed, cond, 1);
            };
            HC_TRY(eg.build(body, "hc_sssp_batched"));
        }
        HC_CUDA_TRY(cudaGraphLaunch(eg.exec, g->stream));
        HC_CUDA_TRY(cudaMemcpyAsync(hctl, b.ctl, sizeof(MsspCtl), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        ::hc::count_launch(2 * kEpochLaunches * ((hctl->epochs + 1) / 2));
    } else {
        for (int ep = 0;; ep++) {
            const auto t0 = std::chrono::steady_clock::now();
            const int c = ep & 1;
            launch_epoch<D, SPL>(g, g->stream, b, c, relaxed, 0, 0);
            ::hc::count_launch(kEpochLaunches);
            HC_CUDA_TRY(cudaGetLastError());
            HC_CUDA_TRY(cudaMemcpyAsync(hctl, b.ctl, sizeof(MsspCtl), cudaMemcpyDeviceToHost, g->stream));
            if (trace) HC_CUDA_TRY(cudaMemcpyAsync(hctl + 1, relaxed, 8, cudaMemcpyDeviceToHost, g->stream));
            HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
            if (trace) {
                const double us =
                    std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
                unsigned long long r = 0;
                std::memcpy(&r, hctl + 1, 8);
                std::fprintf(stderr, "mssp K=%d (%s) epoch %d next %d (%llu edges) relaxed(total) %llu  %.1f us\n", K,
                             D::kPer == 2 ? "16-bit" : "32-bit", ep, hctl->qlen[c ^ 1], hctl->qedges[c ^ 1], r, us);
            }
            if (hctl->stop || hctl->qlen[c ^ 1] == 0) break;
        }
    }
    *fits = true;
    *epochs_out = hctl->epochs;
    if (hctl->stop && hctl->status == kStatusRange) {
        *fits = false;  // 16-bit distances may not hold this group's: the caller reruns it 32-bit
        return HC_OK;
    }
    if (hctl->stop) {
        if (hctl->status == HC_ERR_TIMEOUT) return fail(HC_ERR_TIMEOUT, "hc_sssp_batched: group time limit reached");
        return fail(HC_ERR_NOT_CONVERGED, "hc_sssp_batched: epoch cap reached");
    }
    if (dst || D::kPer == 2) {
        { mssp_transpose<D, SPL><<<grid, 256, 0, g->stream>>>(b.dist, g->N, k, dst, b.ctl); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
    }
    if constexpr (D::kPer == 2) {
        HC_CUDA_TRY(cudaMemcpyAsync(hctl, b.ctl, sizeof(MsspCtl), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        *fits = (int64_t)hctl->maxf + g->w_max < (int64_t)kInf16;
    } else if (dst && (int64_t)g->w_max * std::max<int64_t>(g->n_active - 1, 0) >= (int64_t)kInfDist) {
        // Candidates are clamped at INT32_MAX; when a path of n_active - 1
        // largest weights could reach the clamp, the group's largest finite
        // distance (from the transpose) must stay w_max below it.
        HC_CUDA_TRY(cudaMemcpyAsync(hctl, b.ctl, sizeof(MsspCtl), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        if ((int64_t)hctl->maxf + g->w_max >= (int64_t)kInfDist)
            return fail(HC_ERR_UNSUPPORTED, "hc_sssp_batched: a distance comes within the largest weight (%d) of "
                        "INT32_MAX: int32 distances cannot hold it", g->w_max);
    }
    return HC_OK;
}

// Dispatch on the group's words per lane (16-bit groups stop at 8 words, 512
// sources).
template <class D>
hc_status run_group_spl(int spl, hc_graph *g, const int32_t *h_src, int k, int32_t *dst, int max_epochs,
                        int pull_alpha, bool use_graph, WhileGraph &eg, int *ep, unsigned long long *relaxed,
                        bool *fits) {
    switch (spl) {
        case 1: return run_group<D, 1>(g, h_src, k, dst, max_epochs, pull_alpha, use_graph, eg, ep, relaxed, fits);
        case 2: return run_group<D, 2>(g, h_src, k, dst, max_epochs, pull_alpha, use_graph, eg, ep, relaxed, fits);
        case 4: return run_group<D, 4>(g, h_src, k, dst, max_epochs, pull_alpha, use_graph, eg, ep, relaxed, fits);
        case 8: return run_group<D, 8>(g, h_src, k, dst, max_epochs, pull_alpha, use_graph, eg, ep, relaxed, fits);
        case 16:
            if constexpr (D::kPer == 1)
                return run_group<D, 16>(g, h_src, k, dst, max_epochs, pull_alpha, use_graph, eg, ep, relaxed, fits);
            [[fallthrough]];
        default: return fail(HC_ERR_INVALID_ARG, "hc_sssp_batched: bad group width");
    }
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_sssp_batched(hc_graph *g, const int32_t *sources, int32_t num_sources, int32_t *dist_out,
                                     const hc_batch_opts *opts, hc_batch_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    ReclaimScope reclaim_scope(g, kKeepBatch);
    if (!sources || num_sources < 1) return fail(HC_ERR_INVALID_ARG, "hc_sssp_batched: bad source list");
    if (g->wtype != HC_W_I32) return fail(HC_ERR_UNSUPPORTED, "hc_sssp_batched: graph needs int32 edge weights");
    hc_batch_opts o{};
    if (opts) o = *opts;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (o.dist_bits != 0 && o.dist_bits != 16 && o.dist_bits != 32)
        return fail(HC_ERR_INVALID_ARG, "hc_sssp_batched: dist_bits must be 0, 16 or 32");
    std::vector<int32_t> src(num_sources);
    HC_CUDA_TRY(cudaMemcpy(src.data(), sources, sizeof(int32_t) * num_sources, cudaMemcpyDefault));
    for (int32_t s : src)
        if (s < 0 || s >= g->N) return fail(HC_ERR_INVALID_ARG, "hc_sssp_batched: source %d out of range", s);
    // Weights must be non-negative; pull epochs need symmetric weights; 16-bit
    // distances need weights of at most kMsspNarrowMaxW.
    HC_TRY(ensure_weight_stats(g));
    if (g->w_negative) return fail(HC_ERR_INVALID_ARG, "hc_sssp_batched: negative edge weight");
    const bool narrow_ok = o.dist_bits != 32 && g->w_max <= kMsspNarrowMaxW;
    // Group width: 32, 64, 128, 256 or 512 sources (16-bit distances from 64
    // up).  The default is 512 with 16-bit distances, else 256 (a 1 KB row
    // either way: wider rows read more bytes per edge for no gain per
    // source), halved while the distance matrix would take over 40% of the
    // free device memory or while half the width still holds every source.
    if (o.group <= 0) o.group = g->tune.mssp_group;
    if (o.switch_alpha == 0) o.switch_alpha = g->tune.mssp_switch_alpha;
    int group = o.group <= 32 ? 32 : o.group <= 64 ? 64 : o.group <= 128 ? 128 : o.group <= 256 ? 256 : 512;
    if (o.group <= 0) {
        size_t free_b = 0, total_b = 0;
        HC_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        free_b += g->ws_batch.bytes + g->ws_out0.bytes;  // workspaces are reused
        const double bytes = narrow_ok ? 2.0 : 4.0;
        group = narrow_ok ? 512 : 256;
        while (group > 32 && (double)g->N * group * bytes > 0.4 * (double)free_b) group /= 2;
        const int floor_w = narrow_ok ? 64 : 32;
        while (group > floor_w && group / 2 >= num_sources) group /= 2;
    }
    bool narrow = narrow_ok && group >= 64;
    const int pull_alpha = !g->w_symmetric ? 0 : o.switch_alpha == 0 ? kPullAlpha : std::max(o.switch_alpha, 0);
    if (pull_alpha > 0) HC_TRY(ensure_pull_plan(g));
    const int64_t n = g->N;
    const bool dev_out = is_device_pointer(dist_out);
    if (dist_out && !dev_out) HC_TRY(g->ws_out0.ensure(sizeof(int32_t) * (size_t)group * n));
    // Chaotic relaxation finalises at least one more hop per epoch: N + 1 bounds the loop.
    const int max_epochs = o.max_epochs > 0 ? o.max_epochs : g->N + 1;
    HC_TRY(g->ws_src.ensure(64));
    unsigned long long *relaxed = g->ws_src.as<unsigned long long>();
    HC_CUDA_TRY(cudaMemsetAsync(relaxed, 0, 8, g->stream));
    HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    int epochs_max = 0, groups = 0, wide_groups = 0, reruns = 0;
    // The epoch loop runs as a CUDA graph unless use_graph asks otherwise.
    const bool use_graph = o.use_graph != HC_GRAPH_OFF;
    // Built by the first group of each kind, reused by the others.  Once a
    // group has been rerun with 32-bit words, the rest of the call stays
    // 32-bit (their workspace differs), at most 256 sources per group.
    WhileGraph eg_narrow, eg_wide;
    int wide_width = group;
    for (int s0 = 0; s0 < num_sources;) {
        const int width = narrow ? group : wide_width;
        const int k = std::min(width, num_sources - s0);
        int32_t *dst = nullptr;
        if (dist_out) dst = dev_out ? dist_out + (size_t)s0 * n : g->ws_out0.as<int32_t>();
        int ep = 0;
        bool fits = true;
        if (narrow) {
            HC_TRY(run_group_spl<NarrowDist>(width / 64, g, src.data() + s0, k, dst, max_epochs, pull_alpha, use_graph,
                                             eg_narrow, &ep, relaxed, &fits));
            if (!fits) {
                narrow = false;
                reruns++;
                wide_width = std::min(group, 256);
                continue;  // the same sources again, 32-bit
            }
        } else {
            HC_TRY(run_group_spl<WideDist>(width / 32, g, src.data() + s0, k, dst, max_epochs, pull_alpha, use_graph,
                                           eg_wide, &ep, relaxed, &fits));
            wide_groups++;
        }
        if (dist_out && !dev_out)
            HC_TRY(copy_out(dist_out + (size_t)s0 * n, dst, sizeof(int32_t) * (size_t)k * n, g->stream));
        epochs_max = std::max(epochs_max, ep);
        s0 += k;
        groups++;
    }
    HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    float ms = 0;
    HC_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
    unsigned long long rel = 0;
    HC_CUDA_TRY(cudaMemcpy(&rel, relaxed, 8, cudaMemcpyDeviceToHost));
    if (stats) {
        stats->epochs = epochs_max;
        stats->groups = groups;
        stats->ms = ms;
        // 8 B (neighbour + weight) per edge visit of a row, shared by the
        // group's sources, plus the distance read per source relaxed (2 B
        // for 16-bit distances, 4 B for 32-bit).
        stats->bytes_model = (double)rel / (double)group * 8.0 + (double)rel * (wide_groups ? 4.0 : 2.0);
        stats->wide_groups = wide_groups;
        stats->reruns = reruns;
    }
    return HC_OK;
}
