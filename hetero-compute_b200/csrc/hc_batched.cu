// Batched multi-source BFS (batched SSSP lives in hc_batched_sssp.cu).
//
// The reference runs sources one after another, each a full driver call
// (src/benchmarks/gpu_benchmark.cuh:577-586).  Here a group of sources shares
// every sweep over the CSR.
//
// BFS (bit-sliced frontiers, after Then et al., "The more the merrier:
// efficient multi-source graph traversal", VLDB 2014).  Per vertex, K64 64-bit
// words: `seen` (updated in place by the vertex's owner) and the frontier
// `front` (double-buffered; valid only where the 1-bit activity map is set).
// A level is a pull: next[v] = OR over neighbours u with an active frontier of
// front[u], minus seen[v].
//   - one thread per vertex, so a warp holds 32 consecutive vertices and the
//     depth rows of each source are written 128 bytes at a time;
//   - four neighbours in flight per thread (probe + 8*K64-byte gather each);
//   - a `done` bitmap skips vertices every source has reached;
//   - rows longer than kMsHub edges are cut into kMsTask-edge tasks whose
//     warps OR their partial words into a per-row accumulator; the last task
//     of a row (per-row counter) applies the update.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hc_graph.cuh"

namespace hc {
namespace {

// ------------------------------------------------------------------- BFS

constexpr int kMsHub = 256;   // rows with more edges are split into tasks
constexpr int kMsTask = 256;  // edges per task
constexpr int kMsThreads = 256;

struct MsPlan {
    const int32_t *hub_rows;  // rows with more than kMsHub edges
    const int2 *tasks;        // (hub index, chunk)
    int n_hubs, n_tasks;
};

// Level control in device memory.  The kernels of a level read the level
// number and the push/pull choice from here, so the same launch sequence runs
// from the host loop and as the body of a graph's while node, whose condition
// msbfs_end sets.
struct MsCtl {
    unsigned long long found;   // vertices that gained a frontier bit this level
    unsigned long long fedges;  // edges out of the current frontier
    int ptasks;                 // push tasks queued
    int tlen;                   // touched vertices (push)
    int level;
    int fin;                    // a level found nothing: the traversal is over
    int stop;                   // ended early; status says why
    int status;
    int max_levels;
    int push_alpha;             // push while fedges * push_alpha < m (0: pull only)
    long long m;
    double bytes;               // bytes model, summed over levels
    unsigned long long t0;
};
// Default direction switch: push while the frontier's edges times
// kMsPushAlpha stay below M.
constexpr int kMsPushAlpha = 10;

__device__ __forceinline__ bool ms_live(const MsCtl *c) { return !c->stop && !c->fin; }
__device__ __forceinline__ bool ms_push(const MsCtl *c) {
    return c->push_alpha > 0 && (double)c->fedges * c->push_alpha < (double)c->m;
}

template <int K64>
__device__ __forceinline__ uint64_t full_mask(int word, int nsrc) {
    const int bits = min(64, max(0, nsrc - word * 64));
    return bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
}

template <int K64>
__global__ void msbfs_seed(int nsrc, const int32_t *src, uint64_t *seen, uint64_t *front, uint32_t *act,
                           int32_t *depth, int64_t n) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsrc; s += gridDim.x * blockDim.x) {
        const int32_t v = src[s];
        atomicOr((unsigned long long *)&seen[(size_t)v * K64 + (s >> 6)], 1ull << (s & 63));
        atomicOr((unsigned long long *)&front[(size_t)v * K64 + (s >> 6)], 1ull << (s & 63));
        atomicOr(act + (v >> 5), 1u << (v & 31));
        if (depth) depth[(size_t)s * n + v] = 0;
    }
}

// front words of source-active vertices are gathered only where act has the bit.
template <int K64>
__device__ __forceinline__ void or_front(const uint64_t *front, const uint32_t *act, int32_t u, uint64_t (&acc)[K64]) {
    if ((__ldg(act + (u >> 5)) >> (u & 31)) & 1u) {
        const uint64_t *f = front + (size_t)u * K64;
#pragma unroll
        for (int j = 0; j < K64; j++) acc[j] |= __ldg(f + j);
    }
}

// Writes depth = level for every (source bit, vertex) in nw, one coalesced
// masked store per source with a new bit among the warp's 32 vertices.
template <int K64>
__device__ __forceinline__ void write_depths_warp(const uint64_t (&nw)[K64], int32_t v, bool valid, int32_t *depth,
                                                  int64_t n, int level) {
#pragma unroll
    for (int j = 0; j < K64; j++) {
        uint64_t any = nw[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) any |= __shfl_xor_sync(kFull, any, o);
        while (any) {
            const int b = __ffsll((long long)any) - 1;
            any &= any - 1;
            if (valid && ((nw[j] >> b) & 1ull)) depth[(size_t)(j * 64 + b) * n + v] = level;
        }
    }
}

template <int K64>
__global__ void __launch_bounds__(kMsThreads) msbfs_pull(const int64_t *index, const int32_t *nbr, int32_t n_active,
                                                         int nsrc, uint64_t *seen, const uint64_t *front,
                                                         uint64_t *next, const uint32_t *act, uint32_t *act_next,
                                                         uint32_t *done, int32_t *depth, int64_t n, MsCtl *ctl) {
    if (!ms_live(ctl) || ms_push(ctl)) return;
    const int level = ctl->level;
    unsigned long long *found = &ctl->found;
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long my_found = 0;
    for (int32_t tile = gwarp; tile * 32 < n_active; tile += nwarps) {
        const int32_t v = tile * 32 + lane;
        const uint32_t dw = __ldcg(done + tile);
        bool work = v < n_active && !((dw >> lane) & 1u);
        int64_t b = 0, e = 0;
        if (work) {
            b = index[v];
            e = index[v + 1];
            work = e - b <= kMsHub;  // longer rows: hub tasks
        }
        if (!__any_sync(kFull, work)) continue;
        uint64_t acc[K64];
#pragma unroll
        for (int j = 0; j < K64; j++) acc[j] = 0;
        if (work) {
            int64_t i = b;
            for (; i + 3 < e; i += 4) {
                const int32_t u0 = nbr[i], u1 = nbr[i + 1], u2 = nbr[i + 2], u3 = nbr[i + 3];
                or_front<K64>(front, act, u0, acc);
                or_front<K64>(front, act, u1, acc);
                or_front<K64>(front, act, u2, acc);
                or_front<K64>(front, act, u3, acc);
            }
            for (; i < e; i++) or_front<K64>(front, act, nbr[i], acc);
        }
        uint64_t nw[K64];
        bool any = false, full = true;
        if (work) {
            uint64_t *sv = seen + (size_t)v * K64;
#pragma unroll
            for (int j = 0; j < K64; j++) {
                const uint64_t fm = full_mask<K64>(j, nsrc);
                const uint64_t s = sv[j];
                nw[j] = acc[j] & ~s & fm;
                any |= nw[j] != 0;
                full &= ((s | nw[j]) & fm) == fm;
            }
            if (any) {
                uint64_t *fv = next + (size_t)v * K64;
#pragma unroll
                for (int j = 0; j < K64; j++) {
                    sv[j] |= nw[j];
                    fv[j] = nw[j];
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < K64; j++) nw[j] = 0;
            full = false;
        }
        const unsigned ab = __ballot_sync(kFull, any), fb = __ballot_sync(kFull, work && full);
        if (lane == 0) {
            if (ab) atomicOr(act_next + tile, ab);
            if (fb) atomicOr(done + tile, fb);
            my_found += __popc(ab);
        }
        if (depth && ab) write_depths_warp<K64>(nw, v, work, depth, n, level + 1);
    }
    if (lane == 0 && my_found) atomicAdd(found, my_found);
}

// Hub rows: a warp per (row, chunk); partial words OR into acc[h]; the last
// chunk of the row (counter) applies the update and resets acc / counter.
template <int K64>
__global__ void __launch_bounds__(kMsThreads) msbfs_hub(const int64_t *index, const int32_t *nbr, MsPlan plan,
                                                        int nsrc, uint64_t *seen, const uint64_t *front,
                                                        uint64_t *next, const uint32_t *act, uint32_t *act_next,
                                                        uint32_t *done, uint64_t *hub_acc, unsigned *hub_cnt,
                                                        int32_t *depth, int64_t n, MsCtl *ctl) {
    if (!ms_live(ctl) || ms_push(ctl)) return;
    const int level = ctl->level;
    unsigned long long *found = &ctl->found;
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int t = gwarp; t < plan.n_tasks; t += nwarps) {
        const int2 tk = plan.tasks[t];
        const int32_t r = plan.hub_rows[tk.x];
        if ((__ldcg(done + (r >> 5)) >> (r & 31)) & 1u) continue;  // same answer for every chunk of r
        const int64_t rb = index[r], re = index[r + 1];
        const int64_t b = rb + (int64_t)tk.y * kMsTask, e = min(re, b + (int64_t)kMsTask);
        const int nchunks = (int)((re - rb + kMsTask - 1) / kMsTask);
        uint64_t acc[K64];
#pragma unroll
        for (int j = 0; j < K64; j++) acc[j] = 0;
        for (int64_t i = b + lane; i < e; i += 32) or_front<K64>(front, act, nbr[i], acc);
#pragma unroll
        for (int j = 0; j < K64; j++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[j] |= __shfl_xor_sync(kFull, acc[j], o);
        }
        uint64_t mine = 0;
#pragma unroll
        for (int j = 0; j < K64; j++)
            if (lane == j) mine = acc[j];
        if (lane < K64 && mine) atomicOr((unsigned long long *)&hub_acc[(size_t)tk.x * K64 + lane], mine);
        __threadfence();
        int last = 0;
        if (lane == 0) last = atomicAdd(hub_cnt + tk.x, 1u) == (unsigned)(nchunks - 1);
        last = __shfl_sync(kFull, last, 0);
        if (!last) continue;
        __threadfence();
        uint64_t nw = 0;
        bool full = true;
        if (lane < K64) {
            const uint64_t w = atomicExch((unsigned long long *)&hub_acc[(size_t)tk.x * K64 + lane], 0ull);
            const uint64_t fm = full_mask<K64>(lane, nsrc);
            const uint64_t s = seen[(size_t)r * K64 + lane];
            nw = w & ~s & fm;
            full = ((s | nw) & fm) == fm;
            if (nw) seen[(size_t)r * K64 + lane] = s | nw;
            next[(size_t)r * K64 + lane] = nw;
        }
        const unsigned ab = __ballot_sync(kFull, nw != 0);
        const unsigned fb = __ballot_sync(kFull, lane < K64 && !full);
        if (lane == 0) {
            hub_cnt[tk.x] = 0;
            if (ab) {
                atomicOr(act_next + (r >> 5), 1u << (r & 31));
                atomicAdd(found, 1ull);
            }
            if (!fb) atomicOr(done + (r >> 5), 1u << (r & 31));
        }
        if (depth && lane < K64) {
            uint64_t x = nw;
            while (x) {
                const int bb = __ffsll((long long)x) - 1;
                x &= x - 1;
                depth[(size_t)(lane * 64 + bb) * n + r] = level + 1;
            }
        }
    }
}

// Push levels (sparse frontiers).  The active vertices become (vertex, chunk)
// tasks of kMsPushChunk edges; each edge ORs the source's frontier words, minus
// the target's seen words, into an accumulator x[v] and queues v once per
// level; a finalize pass applies x to seen / next / depth and clears it.
constexpr int kMsPushChunk = 2048;

__global__ void msbfs_push_tasks(const int64_t *index, const uint32_t *act, int32_t n_active, int2 *tasks,
                                 MsCtl *ctl) {
    if (!ms_live(ctl)) return;
    int *ntasks = &ctl->ptasks;
    unsigned long long *fedges = &ctl->fedges;
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long my_e = 0;
    const int words = (n_active + 31) >> 5;
    for (int w = gwarp; w < words; w += nwarps) {
        const uint32_t bits = __ldcg(act + w);
        const int32_t v = w * 32 + lane;
        int nc = 0;
        if ((bits >> lane) & 1u) {
            const int64_t d = index[v + 1] - index[v];
            my_e += (unsigned long long)d;
            nc = (int)((d + kMsPushChunk - 1) / kMsPushChunk);
        }
        int total;
        const int excl = warp_exclusive_scan(nc, &total);
        int base = 0;
        if (lane == 0 && total) base = atomicAdd(ntasks, total);
        base = __shfl_sync(kFull, base, 0);
        for (int c = 0; c < nc; c++) tasks[base + excl + c] = make_int2(v, c);
    }
    my_e = warp_sum(my_e);
    if (lane == 0 && my_e) atomicAdd(fedges, my_e);
}

template <int K64>
__global__ void __launch_bounds__(kMsThreads) msbfs_push(const int64_t *index, const int32_t *nbr, const int2 *tasks,
                                                         const uint64_t *front, const uint64_t *seen, uint64_t *xacc,
                                                         uint32_t *touched, int32_t *tlist, MsCtl *ctl) {
    if (!ms_live(ctl) || !ms_push(ctl)) return;
    int *tlen = &ctl->tlen;
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nt = ctl->ptasks;
    for (int t = gwarp; t < nt; t += nwarps) {
        const int2 tk = tasks[t];
        const int32_t u = tk.x;
        uint64_t fu[K64];
#pragma unroll
        for (int j = 0; j < K64; j++) fu[j] = __ldg(front + (size_t)u * K64 + j);
        const int64_t rb = index[u], re = index[u + 1];
        const int64_t b = rb + (int64_t)tk.y * kMsPushChunk, e = min(re, b + (int64_t)kMsPushChunk);
        for (int64_t i0 = b; i0 < e; i0 += 32) {
            const int64_t i = i0 + lane;
            bool take = false;
            int32_t v = 0;
            if (i < e) {
                v = nbr[i];
                const uint64_t *sv = seen + (size_t)v * K64;
                bool any = false;
#pragma unroll
                for (int j = 0; j < K64; j++) {
                    const uint64_t nw = fu[j] & ~__ldcg(sv + j);
                    if (nw) {
                        atomicOr((unsigned long long *)&xacc[(size_t)v * K64 + j], nw);
                        any = true;
                    }
                }
                if (any) {
                    const uint32_t bit = 1u << (v & 31);
                    take = !(atomicOr(touched + (v >> 5), bit) & bit);
                }
            }
            const unsigned bal = __ballot_sync(kFull, take);
            if (bal) {
                const int leader = __ffs(bal) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(tlen, __popc(bal));
                base = __shfl_sync(kFull, base, leader);
                if (take) tlist[base + __popc(bal & ((1u << lane) - 1u))] = v;
            }
        }
    }
}

template <int K64>
__global__ void msbfs_push_finalize(const int32_t *tlist, int nsrc, uint64_t *seen, uint64_t *xacc, uint64_t *next,
                                    uint32_t *touched, uint32_t *act_next, uint32_t *done, int32_t *depth, int64_t n,
                                    MsCtl *ctl) {
    if (!ms_live(ctl) || !ms_push(ctl)) return;
    const int nt = ctl->tlen;
    const int level = ctl->level;
    unsigned long long *found = &ctl->found;
    unsigned long long my_found = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
        const int32_t v = tlist[i];
        atomicAnd(touched + (v >> 5), ~(1u << (v & 31)));
        bool any = false, full = true;
        uint64_t nw[K64];
#pragma unroll
        for (int j = 0; j < K64; j++) {
            const uint64_t fm = full_mask<K64>(j, nsrc);
            const uint64_t x = xacc[(size_t)v * K64 + j];
            xacc[(size_t)v * K64 + j] = 0;
            const uint64_t s = seen[(size_t)v * K64 + j];
            nw[j] = x & ~s & fm;
            any |= nw[j] != 0;
            full &= ((s | nw[j]) & fm) == fm;
            if (nw[j]) seen[(size_t)v * K64 + j] = s | nw[j];
            next[(size_t)v * K64 + j] = nw[j];
        }
        if (any) {
            atomicOr(act_next + (v >> 5), 1u << (v & 31));
            my_found++;
            if (depth) {
#pragma unroll
                for (int j = 0; j < K64; j++) {
                    uint64_t x = nw[j];
                    while (x) {
                        const int b = __ffsll((long long)x) - 1;
                        x &= x - 1;
                        depth[(size_t)(j * 64 + b) * n + v] = level + 1;
                    }
                }
            }
        }
        if (full) atomicOr(done + (v >> 5), 1u << (v & 31));
    }
    my_found = warp_sum(my_found);
    if ((threadIdx.x & 31) == 0 && my_found) atomicAdd(found, my_found);
}

__global__ void msbfs_ctl_init(MsCtl *ctl, int max_levels, int push_alpha, long long m) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        MsCtl c{};
        c.max_levels = max_levels;
        c.push_alpha = push_alpha;
        c.m = m;
        c.t0 = globaltimer_ns();
        *ctl = c;
    }
}

// Opens a level: clears the next activity bitmap and the level's counters.
__global__ void msbfs_begin(MsCtl *ctl, uint32_t *act_next, int words) {
    if (!ms_live(ctl)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) act_next[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->found = 0;
        ctl->fedges = 0;
        ctl->ptasks = 0;
        ctl->tlen = 0;
    }
}

// Closes a level: adds its bytes to the model, counts it, and decides whether
// another level runs (something found, under the level cap and the time
// bound); inside a graph it sets the while node's condition.
__global__ void msbfs_end(MsCtl *ctl, double pull_bytes, cudaGraphConditionalHandle cond, int use_cond) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    bool go = false;
    if (ms_live(ctl)) {
        const double fe = (double)ctl->fedges;
        ctl->bytes += ms_push(ctl) ? 16.0 * fe / 8.0 + 4.0 * fe : pull_bytes;
        ctl->level++;
        if (ctl->found == 0) {
            ctl->fin = 1;
        } else if (ctl->level >= ctl->max_levels) {
            ctl->stop = 1;
            ctl->status = HC_ERR_NOT_CONVERGED;
        } else if (globaltimer_ns() - ctl->t0 > c_limits.loop_ns) {
            ctl->stop = 1;
            ctl->status = HC_ERR_TIMEOUT;
        } else {
            go = true;
        }
    }
    if (use_cond) cudaGraphSetConditional(cond, go ? 1u : 0u);
}

}  // namespace
}  // namespace hc

using namespace hc;

namespace {

// Hub rows (> kMsHub edges) and their (row, chunk) tasks, built once per graph.
hc_status ensure_ms_plan(hc_graph *g, MsPlan *plan) {
    if (g->ms_hubs >= 0) {
        const size_t b_rows = ((size_t)g->ms_hubs * 4 + 255) / 256 * 256;
        plan->hub_rows = g->ws_plan_ms.as<const int32_t>();
        plan->tasks = reinterpret_cast<const int2 *>(g->ws_plan_ms.as<const char>() + b_rows);
        plan->n_hubs = g->ms_hubs;
        plan->n_tasks = g->ms_tasks;
        return HC_OK;
    }
    const int32_t na = g->n_active;
    std::vector<int64_t> idx((size_t)na + 1);
    HC_CUDA_TRY(cudaMemcpy(idx.data(), g->index.as<int64_t>(), sizeof(int64_t) * ((size_t)na + 1),
                           cudaMemcpyDeviceToHost));
    std::vector<int32_t> rows;
    std::vector<int2> tasks;
    for (int32_t r = 0; r < na; r++) {
        const int64_t d = idx[r + 1] - idx[r];
        if (d > kMsHub) {
            const int nc = (int)((d + kMsTask - 1) / kMsTask);
            for (int c = 0; c < nc; c++) tasks.push_back(make_int2((int)rows.size(), c));
            rows.push_back(r);
        }
    }
    const size_t b_rows = (rows.size() * 4 + 255) / 256 * 256;
    HC_TRY(g->ws_plan_ms.ensure(b_rows + tasks.size() * sizeof(int2) + 256));
    char *p = g->ws_plan_ms.as<char>();
    if (!rows.empty()) HC_CUDA_TRY(cudaMemcpy(p, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice));
    if (!tasks.empty())
        HC_CUDA_TRY(cudaMemcpy(p + b_rows, tasks.data(), tasks.size() * sizeof(int2), cudaMemcpyHostToDevice));
    plan->hub_rows = (const int32_t *)p;
    plan->tasks = (const int2 *)(p + b_rows);
    plan->n_hubs = (int)rows.size();
    plan->n_tasks = (int)tasks.size();
    g->ms_hubs = plan->n_hubs;
    g->ms_tasks = plan->n_tasks;
    return HC_OK;
}

template <int K64>
hc_status run_msbfs(hc_graph *g, const MsPlan &plan, const int32_t *d_src, int nsrc, int32_t *depth,
                    const hc_batch_opts &o, int *levels_out, double *bytes) {
    const int64_t n = g->N;
    const int W = (int)((n + 31) / 32);
    const size_t nk = (size_t)n * K64;
    const size_t hk = (size_t)std::max(plan.n_hubs, 1) * K64;
    const size_t max_ptasks = (size_t)(g->M / kMsPushChunk) + (size_t)n + 64;
    HC_TRY(g->ws_batch.ensure(nk * 8 * 4 + (size_t)W * 4 * 4 + hk * 8 + (size_t)std::max(plan.n_hubs, 1) * 4 +
                              (size_t)n * 4 + max_ptasks * sizeof(int2) + 16384));
    char *p = g->ws_batch.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    uint64_t *seen = (uint64_t *)take(nk * 8);
    uint64_t *fr[2] = {(uint64_t *)take(nk * 8), (uint64_t *)take(nk * 8)};
    uint32_t *act[2] = {(uint32_t *)take((size_t)W * 4), (uint32_t *)take((size_t)W * 4)};
    uint32_t *done = (uint32_t *)take((size_t)W * 4);
    uint64_t *hub_acc = (uint64_t *)take(hk * 8);
    unsigned *hub_cnt = (unsigned *)take((size_t)std::max(plan.n_hubs, 1) * 4);
    uint64_t *xacc = (uint64_t *)take(nk * 8);
    uint32_t *touched = (uint32_t *)take((size_t)W * 4);
    int32_t *tlist = (int32_t *)take((size_t)n * 4);
    int2 *ptasks = (int2 *)take(max_ptasks * sizeof(int2));
    MsCtl *ctl = (MsCtl *)take(sizeof(MsCtl));
    HC_CUDA_TRY(cudaMemsetAsync(xacc, 0, nk * 8, g->stream));
    HC_CUDA_TRY(cudaMemsetAsync(touched, 0, (size_t)W * 4, g->stream));
    HC_CUDA_TRY(cudaMemsetAsync(seen, 0, nk * 8, g->stream));
    HC_CUDA_TRY(cudaMemsetAsync(fr[0], 0, nk * 8, g->stream));  // the seed ORs into it
    HC_CUDA_TRY(cudaMemsetAsync(act[0], 0, (size_t)W * 4, g->stream));
    HC_CUDA_TRY(cudaMemsetAsync(done, 0, (size_t)W * 4, g->stream));
    HC_CUDA_TRY(cudaMemsetAsync(hub_acc, 0, hk * 8, g->stream));
    HC_CUDA_TRY(cudaMemsetAsync(hub_cnt, 0, (size_t)std::max(plan.n_hubs, 1) * 4, g->stream));
    if (depth) HC_CUDA_TRY(cudaMemsetAsync(depth, 0xff, sizeof(int32_t) * (size_t)nsrc * n, g->stream));
    { msbfs_seed<K64><<<(nsrc + 255) / 256, 256, 0, g->stream>>>(nsrc, d_src, seen, fr[0], act[0], depth, n); ::hc::count_launch(); }
    const int max_levels = o.max_epochs > 0 ? o.max_epochs : g->N + 1;
    const int push_alpha = o.switch_alpha == 0 ? kMsPushAlpha : std::max(o.switch_alpha, 0);
    { msbfs_ctl_init<<<1, 32, 0, g->stream>>>(ctl, max_levels, push_alpha, (long long)g->M); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    const int grid = g->sm_count * 8;
    // Offsets + neighbours once per pull level, plus seen / frontier words per vertex.
    const double pull_bytes = 8.0 * (n + 1) + 4.0 * g->M + 3.0 * 8.0 * K64 * (double)g->n_active;
    const int64_t *index = g->index.as<int64_t>();
    const int32_t *nbr = g->nbr.as<int32_t>();
    // One level of parity c: begin, push (tasks, edges, finalize) and pull
    // (hub tasks, rows) kernels, each returning at once when the level is of
    // the other kind, and the end kernel.
    auto launch_level = [&](cudaStream_t st, int c, cudaGraphConditionalHandle cond, int use_cond) {
        msbfs_begin<<<grid, 256, 0, st>>>(ctl, act[c ^ 1], W);
        msbfs_push_tasks<<<grid, kMsThreads, 0, st>>>(index, act[c], g->n_active, ptasks, ctl);
        msbfs_push<K64><<<grid, kMsThreads, 0, st>>>(index, nbr, ptasks, fr[c], seen, xacc, touched, tlist, ctl);
        msbfs_push_finalize<K64><<<grid, kMsThreads, 0, st>>>(tlist, nsrc, seen, xacc, fr[c ^ 1], touched, act[c ^ 1],
                                                              done, depth, n, ctl);
        if (plan.n_tasks > 0)
            msbfs_hub<K64><<<grid, kMsThreads, 0, st>>>(index, nbr, plan, nsrc, seen, fr[c], fr[c ^ 1], act[c],
                                                        act[c ^ 1], done, hub_acc, hub_cnt, depth, n, ctl);
        msbfs_pull<K64><<<grid, kMsThreads, 0, st>>>(index, nbr, g->n_active, nsrc, seen, fr[c], fr[c ^ 1], act[c],
                                                     act[c ^ 1], done, depth, n, ctl);
        msbfs_end<<<1, 32, 0, st>>>(ctl, pull_bytes, cond, use_cond);
    };
    const int per_level = plan.n_tasks > 0 ? 7 : 6;
    HC_TRY(g->pinned.ensure(sizeof(MsCtl) + 64));
    MsCtl *hctl = g->pinned.as<MsCtl>();
    const bool trace = std::getenv("HC_TRACE") != nullptr;
    if (o.use_graph != HC_GRAPH_OFF && !trace) {
        // The graph's body is two levels (parity 0 then 1).
        WhileGraph wg;
        auto body = [&](cudaStream_t cs, cudaGraphConditionalHandle cond) {
            launch_level(cs, 0, cond, 1);
            launch_level(cs, 1, cond, 1);
        };
        HC_TRY(wg.build(body, "hc_bfs_batched"));
        HC_CUDA_TRY(cudaGraphLaunch(wg.exec, g->stream));
        HC_CUDA_TRY(cudaMemcpyAsync(hctl, ctl, sizeof(MsCtl), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        ::hc::count_launch(2 * per_level * ((hctl->level + 1) / 2));
    } else {
        for (int level = 0;; level++) {
            const auto t0 = std::chrono::steady_clock::now();
            launch_level(g->stream, level & 1, 0, 0);
            ::hc::count_launch(per_level);
            HC_CUDA_TRY(cudaGetLastError());
            HC_CUDA_TRY(cudaMemcpyAsync(hctl, ctl, sizeof(MsCtl), cudaMemcpyDeviceToHost, g->stream));
            HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
            if (trace)
                std::fprintf(stderr, "[hc msbfs] L%-3d %s fedges=%-11llu found=%-9llu %8.1f us\n", level,
                             push_alpha > 0 && (double)hctl->fedges * push_alpha < (double)g->M ? "push" : "pull",
                             hctl->fedges,
                             hctl->found,
                             std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count());
            if (hctl->stop || hctl->fin) break;
        }
    }
    if (hctl->stop) {
        if (hctl->status == HC_ERR_TIMEOUT) return fail(HC_ERR_TIMEOUT, "hc_bfs_batched: group time limit reached");
        return fail(HC_ERR_NOT_CONVERGED, "hc_bfs_batched: level cap reached");
    }
    const int level = hctl->level;
    const double b = hctl->bytes;
    *levels_out = level;
    *bytes = b;
    return HC_OK;
}

}  // namespace

extern "C" hc_status hc_bfs_batched(hc_graph *g, const int32_t *sources, int32_t num_sources, int32_t *depth_out,
                                    const hc_batch_opts *opts, hc_batch_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    ReclaimScope reclaim_scope(g, kKeepBatch);
    if (!sources || num_sources < 1) return fail(HC_ERR_INVALID_ARG, "hc_bfs_batched: bad source list");
    hc_batch_opts o{};
    if (opts) o = *opts;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    std::vector<int32_t> src(num_sources);
    HC_CUDA_TRY(cudaMemcpy(src.data(), sources, sizeof(int32_t) * num_sources, cudaMemcpyDefault));
    for (int32_t s : src)
        if (s < 0 || s >= g->N) return fail(HC_ERR_INVALID_ARG, "hc_bfs_batched: source %d out of range", s);
    // Zero fields: the handle's tuned values, else 512-source groups.
    if (o.group <= 0) o.group = g->tune.mbfs_group;
    if (o.switch_alpha == 0) o.switch_alpha = g->tune.mbfs_switch_alpha;
    const int group = o.group > 0 ? std::min(o.group, 512) : 512;
    const int64_t n = g->N;
    const bool dev_out = is_device_pointer(depth_out);
    MsPlan plan{};
    HC_TRY(ensure_ms_plan(g, &plan));
    HC_TRY(g->ws_src.ensure(sizeof(int32_t) * (size_t)num_sources));
    int32_t *d_src = g->ws_src.as<int32_t>();
    HC_CUDA_TRY(cudaMemcpyAsync(d_src, src.data(), sizeof(int32_t) * num_sources, cudaMemcpyHostToDevice, g->stream));
    HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    int max_levels = 0, groups = 0;
    double bytes = 0;
    for (int s0 = 0; s0 < num_sources; s0 += group, groups++) {
        const int k = std::min(group, num_sources - s0);
        int32_t *dep = nullptr;
        if (depth_out) {
            if (dev_out) {
                dep = depth_out + (size_t)s0 * n;
            } else {
                HC_TRY(g->ws_out0.ensure(sizeof(int32_t) * (size_t)k * n));
                dep = g->ws_out0.as<int32_t>();
            }
        }
        int lv = 0;
        double b = 0;
        const int k64 = (k + 63) / 64;
        if (k64 <= 1) HC_TRY(run_msbfs<1>(g, plan, d_src + s0, k, dep, o, &lv, &b));
        else if (k64 <= 2) HC_TRY(run_msbfs<2>(g, plan, d_src + s0, k, dep, o, &lv, &b));
        else if (k64 <= 4) HC_TRY(run_msbfs<4>(g, plan, d_src + s0, k, dep, o, &lv, &b));
        else HC_TRY(run_msbfs<8>(g, plan, d_src + s0, k, dep, o, &lv, &b));
        if (depth_out && !dev_out)
            HC_TRY(copy_out(depth_out + (size_t)s0 * n, dep, sizeof(int32_t) * (size_t)k * n, g->stream));
        max_levels = std::max(max_levels, lv);
        bytes += b;
    }
    HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    float ms = 0;
    HC_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
    if (stats) {
        stats->epochs = max_levels;
        stats->groups = groups;
        stats->bytes_model = bytes;
        stats->ms = ms;
    }
    return HC_OK;
}
