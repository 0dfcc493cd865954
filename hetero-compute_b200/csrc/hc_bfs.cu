// Direction-optimising BFS as one persistent cooperative launch per source.
//
// Reference path: bfs_gpu (src/kernels/gpu/bfs.cuh:21-95) runs bottom-up
// epochs only, one launch + blocking 4-byte D2H + cudaMemset per level; the
// direction heuristic lives in the CPU bfs_do_cpu (src/kernels/cpu/bfs.cuh:48-114,
// alpha = 15, beta = 18).  Here the whole level loop runs on the device: every
// block evaluates the same alpha/beta state machine from counters read after a
// grid barrier, so the per-level selector costs no host round trip.
//
// HBM layout of the working set (W = ceil(N/32) words):
//   depth, parent  int32[N]      outputs (caller's device buffer or ours)
//   visited        uint32[W]     claimed vertices
//   fb[3]          uint32[W]     frontier bitmaps: level L reads fb[L%3],
//                                writes fb[(L+1)%3], zeroes fb[(L+2)%3]
//   q[2]           int32[N]      frontier queues (top-down levels)
//   tasks          int2[]        (vertex, chunk) pieces of long rows
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <mutex>
#include <thread>
#include <vector>

#include "hc_expand.cuh"
#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr int kBfsThreads = 512;
constexpr int kBuSplitLevels = HC_BFS_SPLIT_LEVELS;
constexpr int kTraceLevels = 64;
// Bottom-up levels copy the first kHubWords words of the frontier bitmap
// (the 131072 highest-degree vertices of a degree-sorted graph, which most
// edges point at) into shared memory and probe them there.
constexpr int kHubWords = 4096;
// Every frontier bitmap has a summary: bit i set when one of its words
// [i << sum_shift, (i + 1) << sum_shift) is non-zero, at most kSumWords words,
// so bottom-up levels keep it in shared memory and probe the bitmap in global
// memory only for neighbours whose summary bit is set (on a sparse frontier,
// few: most rows that find no parent stop reading global memory).
constexpr int kSumWords = 4096;

struct LevelCnt {
    int nf;                 // vertices in this frontier
    int tasks;              // long-row tasks queued while expanding it
    unsigned long long mf;  // sum of their degrees (top-down only)
};

struct BfsCtl {
    GridSync gs;
    LevelCnt cnt[3];
    int conv;               // bitmap -> queue conversion counter
    int levels, td_levels, bu_levels;
    unsigned long long vscan, escan, reached;
    struct {
        int mode, nf;
        unsigned long long t_ns;
    } trace[kTraceLevels + 1];  // per-level record for HC_TRACE=1
};

struct BfsArgs {
    const int64_t *index;
    const int32_t *nbr;
    int32_t n, n_active, n_warp_rows;
    int64_t m;
    int32_t *depth, *parent;
    uint32_t *visited, *fb0, *fb1, *fb2;
    uint32_t *sb0, *sb1, *sb2;  // the frontier bitmaps' summaries (sum_words words each)
    int sum_shift, sum_words;
    int32_t *q0, *q1;
    int2 *tasks;
    BfsCtl *ctl;
    int32_t src;
    int alpha, beta, direction, bu_variant, max_levels;
    // Per bottom-up level warp/thread split (the per-epoch granularity
    // selector): bottom-up level k (0 = the first) runs warp per vertex on
    // [0, bu_split[min(k, bu_split_levels - 1)]) and thread per vertex after;
    // bu_split_levels 0 = the fixed split of bu_variant.
    int32_t bu_split[kBuSplitLevels];
    int bu_split_levels;
};

__device__ __forceinline__ uint32_t *fb_sel(const BfsArgs &a, int i) {
    return i == 0 ? a.fb0 : (i == 1 ? a.fb1 : a.fb2);
}
__device__ __forceinline__ uint32_t *sb_sel(const BfsArgs &a, int i) {
    return i == 0 ? a.sb0 : (i == 1 ? a.sb1 : a.sb2);
}

// Sets vertex v's bit in a frontier bitmap and, when its word was empty, the
// word's summary bit.
__device__ __forceinline__ void frontier_add(uint32_t *fb, uint32_t *sb, int cs, int32_t v) {
    const int w = v >> 5;
    if (atomicOr(fb + w, 1u << (v & 31)) == 0u) atomicOr(sb + ((w >> cs) >> 5), 1u << ((w >> cs) & 31));
}

// Word of the frontier bitmap that holds vertex u's bit: the shared copy of
// the hub prefix for u < hub_v, else 0 when u's summary bit (shared) is clear,
// else the bitmap in global memory.  u < 0 (no edge) reads as 0.
__device__ __forceinline__ uint32_t frontier_word_sum(const uint32_t *s_fb, int hub_v, const uint32_t *s_sum, int cs,
                                                      const uint32_t *fb, int32_t u) {
    const bool hub = u >= 0 && u < hub_v;
    const int sw_i = (max(u, 0) >> 5) >> cs;
    const bool need = u >= 0 && !hub && ((s_sum[sw_i >> 5] >> (sw_i & 31)) & 1u);
    const uint32_t hw = s_fb[hub ? (u >> 5) : 0];
    const uint32_t gw = need ? __ldcg(fb + (u >> 5)) : 0u;
    return hub ? hw : gw;
}

// Top-down edge visitor: claim an unvisited neighbour with a CAS on its
// parent, mark it visited and in the next frontier, queue it.
struct TopDownVisit {
    const int64_t *index;
    const int32_t *nbr;
    int32_t *parent, *depth;
    uint32_t *visited, *fnext, *snext;
    int cs;
    int32_t *qnext;
    int *qlen;
    int next_depth;
    unsigned long long mf;  // degree sum of the claimed vertices (this thread)
    struct Item {
        int32_t u, v;
        uint32_t word;
    };
    __device__ __forceinline__ void load(Item &it, int32_t u, int64_t e) {
        it.u = u;
        it.v = nbr[e];
    }
    __device__ __forceinline__ void probe(Item &it) { it.word = __ldcg(visited + (it.v >> 5)); }
    // Stages across the round's items: all CASes in flight, then the marks,
    // then one queue append for the whole warp.
    __device__ __forceinline__ void commit(Item (&it)[kUnroll], const bool (&act)[kUnroll]) {
        bool take[kUnroll];
        int32_t old[kUnroll], v[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; j++) {
            take[j] = act[j] && !((it[j].word >> (it[j].v & 31)) & 1u);
            old[j] = take[j] ? atomicCAS(parent + it[j].v, -1, it[j].u) : 0;
        }
#pragma unroll
        for (int j = 0; j < kUnroll; j++) {
            take[j] = take[j] && old[j] == -1;
            v[j] = take[j] ? it[j].v : 0;
            if (take[j]) {
                const uint32_t bit = 1u << (v[j] & 31);
                depth[v[j]] = next_depth;
                atomicOr(visited + (v[j] >> 5), bit);
                frontier_add(fnext, snext, cs, v[j]);
                mf += (unsigned long long)(index[v[j] + 1] - index[v[j]]);
            }
        }
        warp_append_n(take, v, qnext, qlen);
    }
};

template <bool kStats>
__global__ void __launch_bounds__(kBfsThreads, 2) bfs_persistent(BfsArgs a) {
    __shared__ unsigned long long s_red[32];
    __shared__ uint32_t s_fb[kHubWords];
    __shared__ uint32_t s_sum[kSumWords];
    BfsCtl *ctl = a.ctl;
    const int lane = threadIdx.x & 31;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthreads = gridDim.x * blockDim.x;
    const int gwarp = gtid >> 5, nwarps = nthreads >> 5;
    const int W = (a.n + 31) >> 5;
    const int W_act = (a.n_active + 31) >> 5;

    for (int i = gtid; i < a.n; i += nthreads) {
        a.depth[i] = -1;
        a.parent[i] = -1;
    }
    for (int i = gtid; i < W; i += nthreads) {
        a.visited[i] = 0;
        a.fb0[i] = 0;
        a.fb1[i] = 0;
        a.fb2[i] = 0;
    }
    for (int i = gtid; i < a.sum_words; i += nthreads) {
        a.sb0[i] = 0;
        a.sb1[i] = 0;
        a.sb2[i] = 0;
    }
    const unsigned long long t_start = globaltimer_ns();
    if (!grid_barrier(&ctl->gs)) return;
    if (gtid == 0) {
        const int32_t s = a.src;
        a.depth[s] = 0;
        a.parent[s] = s;
        a.visited[s >> 5] = 1u << (s & 31);
        a.fb0[s >> 5] = 1u << (s & 31);
        a.sb0[((s >> 5) >> a.sum_shift) >> 5] = 1u << (((s >> 5) >> a.sum_shift) & 31);
        a.q0[0] = s;
        ctl->cnt[0].nf = 1;
        ctl->cnt[0].mf = (unsigned long long)(a.index[s + 1] - a.index[s]);
    }
    if (!grid_barrier(&ctl->gs)) return;

    // Direction state (identical in every block).
    bool push = a.direction != 2;
    bool have_queue = true;
    long long edges_to_check = a.m;
    long long num_edges = (long long)(a.index[a.src + 1] - a.index[a.src]);
    unsigned long long my_vscan = 0, my_escan = 0, my_found = 0;
    int L = 0, td_levels = 0, bu_levels = 0;

    for (;;) {
        const int cur = L % 3, nxt = (L + 1) % 3, old = (L + 2) % 3;
        int nf = __ldcg(&ctl->cnt[cur].nf);
        if (nf == 0) break;
        if (L >= a.max_levels) {
            if (gtid == 0) atomicExch(&ctl->gs.err, (int)HC_ERR_NOT_CONVERGED);
            break;
        }
        if (gtid == 0) {
            if (globaltimer_ns() - t_start > c_limits.run_ns) atomicExch(&ctl->gs.err, (int)HC_ERR_TIMEOUT);
            ctl->cnt[old].nf = 0;
            ctl->cnt[old].tasks = 0;
            ctl->cnt[old].mf = 0;
        }
        uint32_t *fcur = fb_sel(a, cur), *fnext = fb_sel(a, nxt), *fold = fb_sel(a, old);
        uint32_t *scur = sb_sel(a, cur), *snext = sb_sel(a, nxt), *sold = sb_sel(a, old);
        for (int i = gtid; i < W_act; i += nthreads) fold[i] = 0;
        for (int i = gtid; i < a.sum_words; i += nthreads) sold[i] = 0;
        int32_t *qcur = (L & 1) ? a.q1 : a.q0;
        int32_t *qnext = (L & 1) ? a.q0 : a.q1;

        if (a.direction == 0 && push && num_edges > edges_to_check / a.alpha) push = false;
        if (gtid == 0 && L < kTraceLevels) {
            ctl->trace[L].mode = push ? 1 : 2;
            ctl->trace[L].nf = nf;
            ctl->trace[L].t_ns = globaltimer_ns();
        }

        if (push) {
            if (!have_queue) {
                // Frontier came from a bottom-up level: compact its bitmap.
                for (int w0 = gwarp * 32; w0 < W_act; w0 += nwarps * 32) {
                    const int w = w0 + lane;
                    uint32_t bits = w < W_act ? __ldcg(fcur + w) : 0u;
                    int total;
                    int pos = warp_exclusive_scan(__popc(bits), &total);
                    int base = 0;
                    if (lane == 0 && total) base = atomicAdd(&ctl->conv, total);
                    pos += __shfl_sync(kFull, base, 0);
                    while (bits) {
                        const int b = __ffs(bits) - 1;
                        bits &= bits - 1;
                        qcur[pos++] = w * 32 + b;
                    }
                }
                if (!grid_barrier(&ctl->gs)) return;
                nf = __ldcg(&ctl->conv);
                have_queue = true;
            }
            edges_to_check -= num_edges;
            td_levels++;
            const int next_depth = L + 1;
            TopDownVisit visit{a.index, a.nbr, a.parent, a.depth, a.visited, fnext, snext, a.sum_shift, qnext,
                               &ctl->cnt[nxt].nf, next_depth, 0ull};
            if (kStats) {
                for (int i = gtid; i < nf; i += nthreads) {
                    const int32_t u = __ldcg(qcur + i);
                    my_escan += (unsigned long long)(a.index[u + 1] - a.index[u]);
                }
                if (gtid == 0) my_vscan += nf;
            }
            expand_small(a.index, qcur, nf, a.tasks, &ctl->cnt[cur].tasks, gwarp, nwarps, visit);
            if (!grid_barrier(&ctl->gs)) return;
            const int nt = __ldcg(&ctl->cnt[cur].tasks);
            if (nt > 0) {
                expand_tasks(a.index, a.tasks, nt, gwarp, nwarps, visit);
            }
            unsigned long long mf_blk = block_sum(visit.mf, s_red);
            if (threadIdx.x == 0 && mf_blk) atomicAdd(&ctl->cnt[nxt].mf, mf_blk);
            if (!grid_barrier(&ctl->gs)) return;
            num_edges = (long long)__ldcg(&ctl->cnt[nxt].mf);
            have_queue = true;
        } else {
            bu_levels++;
            const int next_depth = L + 1;
            int found_local = 0;
            // The frontier bitmap is complete (grid barrier) and read-only in
            // this level: copy its hub prefix.
            const int hub_w = min(kHubWords, W_act);
            const int hub_v = hub_w << 5;
            for (int i = threadIdx.x; i < hub_w; i += blockDim.x) s_fb[i] = __ldcg(fcur + i);
            for (int i = threadIdx.x; i < a.sum_words; i += blockDim.x) s_sum[i] = __ldcg(scur + i);
            __syncthreads();
            const int cs = a.sum_shift;
            // Rows of degree >= 32: warp per vertex, 32 probes per step.
            // AUTO = thread granularity with four probes in flight: on the
            // degree-sorted Kronecker graphs it beats warp-per-row for the
            // >= 32-edge prefix (0.36 vs 0.68 ms per source at scale 22), since
            // the first probes of a sorted row usually hit.  BLOCK selects the
            // warp path only for that prefix.
            const int n_warp = a.bu_split_levels > 0
                                   ? a.bu_split[min(bu_levels - 1, a.bu_split_levels - 1)]
                                   : a.bu_variant == HC_VARIANT_WARP
                                         ? a.n_active
                                         : (a.bu_variant == HC_VARIANT_BLOCK ? a.n_warp_rows : 0);
            const int n_warp_al = min(((n_warp + 31) >> 5) << 5, W_act << 5);
            for (int v = gwarp; v < n_warp_al; v += nwarps) {
                if (v >= a.n_active) break;
                const uint32_t bit = 1u << (v & 31);
                if (__ldcg(a.visited + (v >> 5)) & bit) continue;
                const int64_t b = a.index[v], e = a.index[v + 1];
                int32_t par = -1;
                int64_t probes = 0;
                for (int64_t e0 = b; e0 < e; e0 += 32) {
                    const int64_t i = e0 + lane;
                    bool hit = false;
                    int32_t u = 0;
                    if (i < e) {
                        u = a.nbr[i];
                        hit = (frontier_word_sum(s_fb, hub_v, s_sum, cs, fcur, u) >> (u & 31)) & 1u;
                    }
                    const unsigned bal = __ballot_sync(kFull, hit);
                    if (kStats) probes += bal ? (int64_t)__ffs(bal) : ((e - e0) < 32 ? (e - e0) : (int64_t)32);
                    if (bal) {
                        par = __shfl_sync(kFull, u, __ffs(bal) - 1);
                        break;
                    }
                }
                if (kStats && lane == 0) {
                    my_vscan++;
                    my_escan += probes;
                }
                if (par >= 0 && lane == 0) {
                    a.parent[v] = par;
                    a.depth[v] = next_depth;
                    atomicOr(a.visited + (v >> 5), bit);
                    frontier_add(fnext, snext, cs, v);
                    found_local++;
                }
            }
            // Remaining rows: thread per vertex, warp owns one bitmap word.
            for (int w = (n_warp_al >> 5) + gwarp; w < W_act; w += nwarps) {
                const uint32_t vis = __ldcg(a.visited + w);
                const int v = w * 32 + lane;
                int32_t par = -1;
                if (v < a.n_active && !((vis >> lane) & 1u)) {
                    const int64_t b = a.index[v], e = a.index[v + 1];
                    // Four probes in flight per round; any frontier neighbour is a valid parent.
                    for (int64_t i = b; i < e && par < 0; i += 4) {
                        int32_t u[4];
                        uint32_t wd[4];
#pragma unroll
                        for (int j = 0; j < 4; j++) u[j] = i + j < e ? a.nbr[i + j] : -1;
#pragma unroll
                        for (int j = 0; j < 4; j++) wd[j] = frontier_word_sum(s_fb, hub_v, s_sum, cs, fcur, u[j]);
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            if (par < 0 && u[j] >= 0 && ((wd[j] >> (u[j] & 31)) & 1u)) {
                                par = u[j];
                                if (kStats) my_escan += (unsigned long long)(i + j - b + 1);
                            }
                    }
                    if (kStats) {
                        my_vscan++;
                        if (par < 0) my_escan += (unsigned long long)(e - b);
                    }
                }
                const unsigned bal = __ballot_sync(kFull, par >= 0);
                if (par >= 0) {
                    a.parent[v] = par;
                    a.depth[v] = next_depth;
                }
                if (lane == 0) {
                    fnext[w] = bal;
                    if (bal) {
                        a.visited[w] = vis | bal;
                        atomicOr(snext + ((w >> cs) >> 5), 1u << ((w >> cs) & 31));
                    }
                    found_local += __popc(bal);
                }
            }
            unsigned long long f_blk = block_sum((unsigned long long)found_local, s_red);
            if (threadIdx.x == 0 && f_blk) atomicAdd((unsigned long long *)&ctl->reached, f_blk);
            if (threadIdx.x == 0 && f_blk) atomicAdd(&ctl->cnt[nxt].nf, (int)f_blk);
            if (gtid == 0) ctl->conv = 0;
            if (!grid_barrier(&ctl->gs)) return;
            const int nf_next = __ldcg(&ctl->cnt[nxt].nf);
            if (a.direction == 0 && !(nf_next > nf || nf_next > a.n / a.beta)) {
                push = true;
                num_edges = 1;
            }
            have_queue = false;
        }
        (void)my_found;
        L++;
    }

    if (kStats) {
        unsigned long long v = block_sum(my_vscan, s_red);
        if (threadIdx.x == 0 && v) atomicAdd(&ctl->vscan, v);
        unsigned long long e = block_sum(my_escan, s_red);
        if (threadIdx.x == 0 && e) atomicAdd(&ctl->escan, e);
    }
    if (gtid == 0) {
        ctl->levels = L;
        ctl->trace[L < kTraceLevels ? L : kTraceLevels].t_ns = globaltimer_ns();
        ctl->td_levels = td_levels;
        ctl->bu_levels = bu_levels;
    }
}

// Discovered count for top-down levels is the queue length; add it up after
// the run from the per-level counters is not possible (they rotate), so the
// reached total is recounted from the depth array.
__global__ void count_reached(const int32_t *depth, int32_t n, unsigned long long *out) {
    __shared__ unsigned long long s_red[32];
    unsigned long long c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        c += depth[i] >= 0;
    c = block_sum(c, s_red);
    if (threadIdx.x == 0 && c) atomicAdd(out, c);
}

// Host outputs on a degree-sorted graph: the vertices [n_copy, n) have no
// edges, so every run leaves their depth and parent at -1 (a source among
// them aside: depth 0, parent itself).  A few host threads write those
// suffixes while the GPU runs, and only the first n_copy entries of each
// source's rows cross PCIe.  The threads are joined by the destructor, on
// every return path.
struct SuffixFill {
    std::vector<std::thread> th;
    void start(int32_t *depth, int32_t *parent, const std::vector<int32_t> &src, int64_t n, int64_t n_copy) {
        const int k = (int)src.size();
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int nt = std::max(1, std::min({(int)(hw / 2), 8, k}));
        auto part = [=, &src](int t) {
            for (int i = t; i < k; i += nt) {
                for (int32_t *out : {depth, parent}) {
                    if (!out) continue;
                    // -1 in every byte is -1 in every int32; a large memset streams its
                    // stores without reading the lines first.
                    std::memset(out + (size_t)i * n + n_copy, 0xFF, sizeof(int32_t) * (size_t)(n - n_copy));
                }
                const int32_t s = src[i];
                if (s >= n_copy) {
                    if (depth) depth[(size_t)i * n + s] = 0;
                    if (parent) parent[(size_t)i * n + s] = s;
                }
            }
        };
        for (int t = 0; t < nt; t++) {
            try {
                th.emplace_back(part, t);
            } catch (...) {  // no thread to be had: this share runs here (nothing throws past the C ABI)
                part(t);
            }
        }
    }
    ~SuffixFill() {
        for (auto &t : th) t.join();
    }
};

// Results of the runs of one call, folded on the device after each run so
// that the host need not wait for each source: the first failure (status and
// source), the deepest run, the top-down / bottom-up level counts.
struct BfsFold {
    int err, err_src, levels, td_levels, bu_levels, pad;
};

// Folds the run just finished into *f, then clears the control block for the
// next run (one block).
__global__ void bfs_fold_clear(BfsCtl *ctl, BfsFold *f, int32_t src) {
    if (threadIdx.x == 0) {
        if (ctl->gs.err && !f->err) {
            f->err = ctl->gs.err;
            f->err_src = src;
        }
        f->levels = max(f->levels, ctl->levels);
        f->td_levels += ctl->td_levels;
        f->bu_levels += ctl->bu_levels;
    }
    __syncthreads();
    uint32_t *w = reinterpret_cast<uint32_t *>(ctl);
    for (int i = threadIdx.x; i < (int)(sizeof(BfsCtl) / 4); i += blockDim.x) w[i] = 0u;
}

template <bool kStats>
hc_status launch_bfs(hc_graph *g, const BfsArgs &args) {
    static int blocks_per_sm[2] = {0, 0};
    int &bps = blocks_per_sm[kStats ? 1 : 0];
    if (bps == 0) {
        HC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, bfs_persistent<kStats>, kBfsThreads, 0));
        if (bps < 1) return fail(HC_ERR_CUDA, "BFS kernel cannot be resident");
    }
    dim3 grid(g->sm_count * bps), block(kBfsThreads);
    BfsArgs a = args;
    void *params[] = {&a};
    ::hc::count_launch();
    HC_CUDA_TRY(cudaLaunchCooperativeKernel((void *)bfs_persistent<kStats>, grid, block, params, 0, g->stream));
    return HC_OK;
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_bfs(hc_graph *g, const int32_t *sources, int32_t num_sources, int32_t *depth_out,
                            int32_t *parent_out, const hc_bfs_opts *opts, hc_bfs_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    if (!sources || num_sources < 0) return fail(HC_ERR_INVALID_ARG, "hc_bfs: bad source list");
    hc_bfs_opts o{};
    if (opts) o = *opts;
    // Zero fields: the handle's tuned values, else Beamer's alpha = 15, beta = 18.
    if (o.alpha <= 0) o.alpha = g->tune.bfs_alpha > 0 ? g->tune.bfs_alpha : 15;
    if (o.beta <= 0) o.beta = g->tune.bfs_beta > 0 ? g->tune.bfs_beta : 18;
    // AUTO: the handle's per-level split table when the autotuner left one,
    // else its tuned variant.
    const bool by_level = o.bu_variant == HC_VARIANT_AUTO && g->tune.bfs_bu_split_levels > 0;
    if (o.bu_variant == HC_VARIANT_AUTO) o.bu_variant = (hc_variant)g->tune.bfs_bu_variant;
    if (o.direction < 0 || o.direction > 2) return fail(HC_ERR_INVALID_ARG, "hc_bfs: direction must be 0, 1 or 2");
    if (stats) std::memset(stats, 0, sizeof(*stats));

    std::vector<int32_t> src(num_sources);
    HC_CUDA_TRY(cudaMemcpy(src.data(), sources, sizeof(int32_t) * num_sources, cudaMemcpyDefault));
    for (int32_t s : src)
        if (s < 0 || s >= g->N) return fail(HC_ERR_INVALID_ARG, "hc_bfs: source %d outside [0, %d)", s, g->N);

    const int64_t n = g->N;
    const int64_t W = (n + 31) / 32;
    const int64_t ntasks = max_expand_tasks(g->M, n);
    int sum_shift = 0;
    while (((W + (1ll << sum_shift) - 1) >> sum_shift) > (int64_t)kSumWords * 32) sum_shift++;
    const int sum_words = (int)((((W + (1ll << sum_shift) - 1) >> sum_shift) + 31) / 32);
    const size_t bytes = sizeof(uint32_t) * 4 * W + sizeof(int32_t) * 2 * n + sizeof(int2) * ntasks +
                         3 * (sizeof(uint32_t) * (size_t)sum_words + 256) + 1024;
    HC_TRY(g->ws_bfs.ensure(bytes));
    HC_TRY(g->ws_ctl.ensure(4096));
    char *p = g->ws_bfs.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    BfsArgs a{};
    a.index = g->index.as<int64_t>();
    a.nbr = g->nbr.as<int32_t>();
    a.n = g->N;
    a.n_active = g->n_active;
    a.n_warp_rows = g->n_warp_rows;
    a.m = g->M;
    a.visited = (uint32_t *)take(4 * W);
    a.fb0 = (uint32_t *)take(4 * W);
    a.fb1 = (uint32_t *)take(4 * W);
    a.fb2 = (uint32_t *)take(4 * W);
    a.sb0 = (uint32_t *)take(4 * (size_t)sum_words);
    a.sb1 = (uint32_t *)take(4 * (size_t)sum_words);
    a.sb2 = (uint32_t *)take(4 * (size_t)sum_words);
    a.sum_shift = sum_shift;
    a.sum_words = sum_words;
    a.q0 = (int32_t *)take(4 * n);
    a.q1 = (int32_t *)take(4 * n);
    a.tasks = (int2 *)take(sizeof(int2) * ntasks);
    a.ctl = g->ws_ctl.as<BfsCtl>();
    a.alpha = o.alpha;
    a.beta = o.beta;
    a.direction = o.direction;
    a.bu_variant = (int)o.bu_variant;
    a.max_levels = g->N + 1;
    a.bu_split_levels = 0;
    if (by_level) {
        a.bu_split_levels = std::min(g->tune.bfs_bu_split_levels, kBuSplitLevels);
        for (int k = 0; k < a.bu_split_levels; k++)
            a.bu_split[k] = std::max(0, std::min(g->tune.bfs_bu_split[k], g->n_active));
    }

    const bool dev_depth = is_device_pointer(depth_out);
    const bool dev_parent = is_device_pointer(parent_out);
    if (!depth_out) HC_TRY(g->ws_out0.ensure(4 * n));
    if (!parent_out) HC_TRY(g->ws_out1.ensure(4 * n));
    // Host outputs: staged on the device and copied while the next source runs.
    const bool host_depth = depth_out && !dev_depth, host_parent = parent_out && !dev_parent;
    OutPipe pipe;
    SuffixFill fill;  // declared after the pipe: its threads are joined first on any return
    if (host_depth || host_parent) {
        HC_TRY(pipe.init(g, 2, 4 * n));
        const int64_t n_copy = g->degree_sorted ? (int64_t)g->n_active : n;
        if (n_copy < n) {
            pipe.copy_bytes = sizeof(int32_t) * (size_t)n_copy;
            fill.start(host_depth ? depth_out : nullptr, host_parent ? parent_out : nullptr, src, n, n_copy);
        }
    }

    double total_ms = 0;
    // Without per-run statistics or a trace the runs go back to back: each
    // run's result is folded on the device and the host waits once, at the
    // end (with them, it reads each run's control block after it).
    const bool per_run = (o.collect_stats && stats) || std::getenv("HC_TRACE");
    static_assert(sizeof(BfsCtl) + 64 <= 2048, "BfsCtl overlaps the fold record");
    BfsFold *fold = reinterpret_cast<BfsFold *>(reinterpret_cast<char *>(a.ctl) + 2560);
    if (!per_run) {
        HC_TRY(ctl_zero(g, fold, sizeof(BfsFold)));
        HC_TRY(ctl_zero(g, a.ctl, sizeof(BfsCtl)));
        HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    }
    for (int32_t i = 0; i < num_sources; i++) {
        a.src = src[i];
        int32_t *stage[2] = {nullptr, nullptr};
        if (host_depth || host_parent) HC_TRY(pipe.acquire(i, stage));
        a.depth = dev_depth ? depth_out + (size_t)i * n : host_depth ? stage[0] : g->ws_out0.as<int32_t>();
        a.parent = dev_parent ? parent_out + (size_t)i * n : host_parent ? stage[1] : g->ws_out1.as<int32_t>();
        if (!per_run) {
            HC_TRY(launch_bfs<false>(g, a));
            if (host_depth || host_parent) {
                void *dst[2] = {host_depth ? (void *)(depth_out + (size_t)i * n) : nullptr,
                                host_parent ? (void *)(parent_out + (size_t)i * n) : nullptr};
                HC_TRY(pipe.release(i, dst));
            }
            { bfs_fold_clear<<<1, 256, 0, g->stream>>>(a.ctl, fold, a.src); ::hc::count_launch(); }
            HC_CUDA_TRY(cudaGetLastError());
            continue;
        }
        HC_TRY(ctl_zero(g, a.ctl, sizeof(BfsCtl)));
        HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
        HC_TRY(o.collect_stats ? launch_bfs<true>(g, a) : launch_bfs<false>(g, a));
        HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
        if (host_depth || host_parent) {
            void *dst[2] = {host_depth ? (void *)(depth_out + (size_t)i * n) : nullptr,
                            host_parent ? (void *)(parent_out + (size_t)i * n) : nullptr};
            HC_TRY(pipe.release(i, dst));
        }
        static_assert(sizeof(BfsCtl) <= kCtlSlotBytes, "BfsCtl exceeds a control-read slot");
        BfsCtl c;
        const void *h_ctl = nullptr, *h_cnt = nullptr;
        HC_TRY(ctl_read(g, a.ctl, sizeof(c), 0, &h_ctl));
        if (o.collect_stats && stats) {
            unsigned long long *cnt = (unsigned long long *)((char *)a.ctl + 2048);
            HC_TRY(ctl_zero(g, cnt, 8));
            { count_reached<<<g->sm_count * 4, 256, 0, g->stream>>>(a.depth, g->N, cnt); ::hc::count_launch(); }
            HC_TRY(ctl_read(g, cnt, 8, 1, &h_cnt));
        }
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        std::memcpy(&c, h_ctl, sizeof(c));
        if (h_cnt) {
            unsigned long long reached = 0;
            std::memcpy(&reached, h_cnt, 8);
            stats->reached += (int32_t)reached;
        }
        if (c.gs.err) return fail((hc_status)c.gs.err, "hc_bfs: device run from source %d ended with status %d",
                                  src[i], c.gs.err);
        float ms = 0;
        HC_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
        total_ms += ms;
        if (stats) {
            stats->levels = std::max(stats->levels, c.levels);
            stats->td_levels += c.td_levels;
            stats->bu_levels += c.bu_levels;
            stats->vertices_scanned += (int64_t)c.vscan;
            stats->edges_scanned += (int64_t)c.escan;
        }
        if (std::getenv("HC_TRACE")) {
            const int nl = std::min(c.levels, kTraceLevels);
            std::fprintf(stderr, "[hc bfs] src %d: %d levels, %.1f us\n", src[i], c.levels, ms * 1e3);
            for (int l = 0; l < nl; l++)
                std::fprintf(stderr, "[hc bfs]   L%-3d %s nf=%-9d %8.1f us\n", l, c.trace[l].mode == 1 ? "TD" : "BU",
                             c.trace[l].nf, (c.trace[l + 1].t_ns - c.trace[l].t_ns) * 1e-3);
        }
    }
    if (!per_run) {
        HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
        const void *h_fold = nullptr;
        HC_TRY(ctl_read(g, fold, sizeof(BfsFold), 0, &h_fold));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        BfsFold f;
        std::memcpy(&f, h_fold, sizeof(f));
        if (f.err) return fail((hc_status)f.err, "hc_bfs: device run from source %d ended with status %d",
                               f.err_src, f.err);
        float ms = 0;
        HC_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
        total_ms = ms;
        if (stats) {
            stats->levels = f.levels;
            stats->td_levels = f.td_levels;
            stats->bu_levels = f.bu_levels;
        }
    }
    if (host_depth || host_parent) HC_TRY(pipe.finish());
    if (stats) {
        stats->ms = total_ms;
        // Streamed bytes: 16 B offsets per scanned vertex, 4 B per scanned edge,
        // 4 B per discovered vertex, and for bottom-up levels two bitmap sweeps.
        stats->bytes_model = 16.0 * (double)stats->vertices_scanned + 4.0 * (double)stats->edges_scanned +
                             4.0 * (double)stats->reached +
                             2.0 * ((double)g->N / 8.0) * (double)stats->bu_levels;
    }
    return HC_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free BFS.
//
// Some callers cannot allocate device memory at the moment they need a BFS:
// code running inside another framework's caching allocator or memory pool
// (where a cudaMalloc would bypass or fragment the pool), paths that must not
// trigger the implicit device synchronisation a cudaMalloc / cudaFree can
// cause, and hosts that pre-plan every byte of HBM.  hc_bfs_noalloc serves
// them: the caller passes the graph and the outputs in its own device memory,
// and the working set (visited and frontier bitmaps, the two queues, the
// long-row task list and the control block) lives in one fixed file-scope
// device array, g_bfs_scratch, sized for graphs of up to kNoAllocMaxNodes
// vertices and kNoAllocMaxEdges edges (about 13 MB, held by every GPU that
// loads this library until the process exits).  It runs the same persistent
// direction-optimising kernel as hc_bfs.
namespace hc {
namespace {

constexpr int32_t kNoAllocMaxNodes = 1 << 20;
constexpr int64_t kNoAllocMaxEdges = 1ll << 24;
constexpr size_t na_align(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kNaWords = (size_t)kNoAllocMaxNodes / 32;
constexpr size_t kNaTasks = (size_t)(kNoAllocMaxEdges / kTaskEdges + kNoAllocMaxEdges / (kSmallDeg + 1) + 64);
// Frontier summaries: one bit per bitmap word (kNaWords <= 32 * kSumWords).
constexpr size_t kNaSumWords = (kNaWords + 31) / 32;
static_assert(kNaWords <= (size_t)kSumWords * 32, "summary of the fixed-size bitmaps needs a shift");
constexpr size_t kNoAllocBytes = na_align(sizeof(BfsCtl)) + na_align(sizeof(int)) + 4 * na_align(4 * kNaWords) +
                                 3 * na_align(4 * kNaSumWords) + 2 * na_align(4 * (size_t)kNoAllocMaxNodes) +
                                 na_align(sizeof(int2) * kNaTasks);

static __device__ __align__(256) unsigned char g_bfs_scratch[kNoAllocBytes];

// In host code g_bfs_scratch names a host-side shadow, not device memory: the
// device address comes from cudaGetSymbolAddress, once per device, with that
// device current, and is cached here.
constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
void *g_na_addr[kNaMaxDevices] = {};

hc_status noalloc_scratch(int dev, unsigned char **out) {
    if (dev < 0 || dev >= kNaMaxDevices) return fail(HC_ERR_UNSUPPORTED, "hc_bfs_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_bfs_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(HC_ERR_CUDA, "hc_bfs_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        }
        g_na_addr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_na_addr[dev]);
    return HC_OK;
}

bool on_device(const void *p, int dev) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) && attr.device == dev;
}

}  // namespace
}  // namespace hc

extern "C" hc_status hc_bfs_noalloc(const int64_t *index, const int32_t *neighbors, int32_t num_nodes,
                                    int64_t num_edges, int32_t source, int32_t *depth_out, int32_t *parent_out,
                                    void *stream) {
    using namespace hc;
    clear_error();
    if (num_nodes < 1 || num_nodes > kNoAllocMaxNodes || num_edges < 0 || num_edges > kNoAllocMaxEdges)
        return fail(HC_ERR_INVALID_ARG,
                    "hc_bfs_noalloc: graph of %d vertices / %lld edges exceeds the fixed working set "
                    "(at most %d vertices and %lld edges); use hc_bfs",
                    num_nodes, (long long)num_edges, kNoAllocMaxNodes, (long long)kNoAllocMaxEdges);
    if (source < 0 || source >= num_nodes)
        return fail(HC_ERR_INVALID_ARG, "hc_bfs_noalloc: source %d outside [0, %d)", source, num_nodes);
    int dev = 0;
    HC_CUDA_TRY(cudaGetDevice(&dev));
    if (!index || !neighbors || !depth_out || !parent_out || !on_device(index, dev) ||
        (num_edges > 0 && !on_device(neighbors, dev)) || !on_device(depth_out, dev) || !on_device(parent_out, dev))
        return fail(HC_ERR_INVALID_ARG,
                    "hc_bfs_noalloc: index, neighbors, depth_out and parent_out must be device memory of the "
                    "current device");
    unsigned char *base = nullptr;
    HC_TRY(noalloc_scratch(dev, &base));
    int sms = 0, bps = 0;
    HC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, bfs_persistent<false>, kBfsThreads, 0));
    if (bps < 1) return fail(HC_ERR_CUDA, "hc_bfs_noalloc: BFS kernel cannot be resident");

    unsigned char *p = base;
    auto take = [&](size_t b) {
        unsigned char *r = p;
        p += na_align(b);
        return r;
    };
    BfsArgs a{};
    a.ctl = reinterpret_cast<BfsCtl *>(take(sizeof(BfsCtl)));
    int *check_flag = reinterpret_cast<int *>(take(sizeof(int)));
    a.visited = reinterpret_cast<uint32_t *>(take(4 * kNaWords));
    a.fb0 = reinterpret_cast<uint32_t *>(take(4 * kNaWords));
    a.fb1 = reinterpret_cast<uint32_t *>(take(4 * kNaWords));
    a.fb2 = reinterpret_cast<uint32_t *>(take(4 * kNaWords));
    a.sb0 = reinterpret_cast<uint32_t *>(take(4 * kNaSumWords));
    a.sb1 = reinterpret_cast<uint32_t *>(take(4 * kNaSumWords));
    a.sb2 = reinterpret_cast<uint32_t *>(take(4 * kNaSumWords));
    a.sum_shift = 0;
    a.sum_words = (int)((((num_nodes + 31) / 32) + 31) / 32);
    a.q0 = reinterpret_cast<int32_t *>(take(4 * (size_t)kNoAllocMaxNodes));
    a.q1 = reinterpret_cast<int32_t *>(take(4 * (size_t)kNoAllocMaxNodes));
    a.tasks = reinterpret_cast<int2 *>(take(sizeof(int2) * kNaTasks));
    a.index = index;
    a.nbr = neighbors;
    a.n = num_nodes;
    a.n_active = num_nodes;  // no degree analysis here: scan every vertex
    a.n_warp_rows = 0;
    a.m = num_edges;
    a.depth = depth_out;
    a.parent = parent_out;
    a.src = source;
    a.alpha = 15;
    a.beta = 18;
    a.direction = 0;
    a.bu_variant = HC_VARIANT_THREAD;
    a.max_levels = num_nodes + 1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The caller's CSR is checked before the traversal reads it (offsets
    // rising from 0 to num_edges, neighbour ids in [0, num_nodes)); the check
    // writes its flag into the fixed array too.
    HC_TRY(csr_check_async(index, neighbors, 1, num_nodes, num_edges, check_flag, sms, s));
    int bad = 0;
    HC_CUDA_TRY(cudaMemcpyAsync(&bad, check_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    HC_CUDA_TRY(cudaStreamSynchronize(s));
    if (bad & 1) return fail(HC_ERR_INVALID_ARG, "hc_bfs_noalloc: offsets must rise from 0 to num_edges");
    if (bad & 2) return fail(HC_ERR_INVALID_ARG, "hc_bfs_noalloc: neighbour id outside [0, num_nodes)");
    // The array keeps the previous call's contents; the control block must
    // start at zero (the kernel initialises everything else it reads).
    HC_CUDA_TRY(cudaMemsetAsync(a.ctl, 0, sizeof(BfsCtl), s));
    void *params[] = {&a};
    ::hc::count_launch();
    HC_CUDA_TRY(cudaLaunchCooperativeKernel((void *)bfs_persistent<false>, dim3(sms * bps), dim3(kBfsThreads), params,
                                            0, s));
    int err = 0;
    HC_CUDA_TRY(cudaMemcpyAsync(&err, &a.ctl->gs.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    HC_CUDA_TRY(cudaStreamSynchronize(s));
    if (err) return fail((hc_status)err, "hc_bfs_noalloc: device run ended with status %d", err);
    return HC_OK;
}
