// PageRank in the reference's sweep order, bit for bit.
//
// pr_pull_cpu (src/kernels/cpu/pr.cuh:33-65) with epoch_pr_pull_cpu_one_to_one
// (src/kernels/cpu/pr.cuh:157-187), run on one thread, updates the scores in
// place from vertex 0 to N-1: vertex v sums score[u] / deg(u) over its row in
// CSR order, so it sees this sweep's new score for every neighbour u < v and
// the previous sweep's score for every neighbour u > v, and it stores
// base + d * sum only when that moves the score by more than 5e-8.  The
// reference's GPU driver (src/kernels/gpu/pr.cuh:42-118) applies the same rule
// in whatever order its threads run, so its scores vary from run to run; the
// single-thread CPU order is the one deterministic result it has.
//
// On a graph whose edges all have a reverse, that order is reproduced exactly
// by a level schedule: level(v) = 1 + max level(u) over the neighbours u < v
// (0 when there is none).  Every lower neighbour of v sits in an earlier level
// and every higher neighbour in a later one, and the vertices of one level
// share no edge, so updating a level's vertices in parallel, level after
// level, reads exactly the values the sequential sweep reads.  Each row is
// summed in CSR order with the same fp32 operations (explicit round-to-nearest
// intrinsics, no multiply-add contraction): the scores equal the reference's
// single-thread output bit for bit.
//
// The schedule (vertex order grouped by level, and level offsets) is built
// once per graph by Kahn's algorithm on the device: count each vertex's lower
// neighbours, start from the vertices with none, and release a vertex when its
// last lower neighbour has been placed.  A cooperative persistent kernel then
// runs the sweeps with a grid barrier after each level and the per-sweep
// update count read after the last barrier.  A lane sums a short row by
// itself; the warp sums a long row together (its lanes gather 32 terms at a
// time and every lane adds them in row order from shuffles).  Either way each
// sum is the sequential one.
#include <algorithm>
#include <vector>

#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr int kOrdThreads = 256;
constexpr int kSweepsPerLaunch = 8;
// Rows up to this many edges are summed by one lane from terms the warp
// gathered into shared memory (32 rows' worth at most kShortRow * 32 terms);
// longer ones by the whole warp, kLongDepth 32-term chunks in flight.
constexpr int kShortRow = 32;
constexpr int kGatherUnroll = 4;
constexpr int kLongDepth = 8;

// cnt[x] = neighbours u < x in x's row; vertices with none open level 0.
__global__ void ord_count_lower(const int64_t *index, const int32_t *nbr, int32_t n, int32_t *cnt,
                                int32_t *order, int32_t *tail) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; x < n; x += nw) {
        const int64_t b = index[x], e = index[x + 1];
        int c = 0;
        for (int64_t i = b + lane; i < e; i += 32) c += nbr[i] < x;
        c = warp_sum(c);
        if (lane == 0) {
            cnt[x] = c;
            if (c == 0) order[atomicAdd(tail, 1)] = x;
        }
    }
}

// Places the vertices of level [lo, hi): each releases its higher neighbours,
// and a neighbour whose count reaches zero joins the next level.
__global__ void ord_expand(const int64_t *index, const int32_t *nbr, int32_t *order, int32_t lo, int32_t hi,
                           int32_t *cnt, int32_t *tail) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = lo + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < hi; i += nw) {
        const int32_t x = order[i];
        const int64_t b = index[x], e = index[x + 1];
        for (int64_t j = b + lane; j < e; j += 32) {
            const int32_t u = nbr[j];
            if (u > x && atomicSub(&cnt[u], 1) == 1) order[atomicAdd(tail, 1)] = u;
        }
    }
}

__global__ void ord_init(int32_t n, const int64_t *index, const float *init, float *score, float *gv, float *degf) {
    const float x0 = __fdiv_rn(1.0f, __int2float_rn(n));
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        // deg as float, the conversion `score[u] / g.get_degree(u)` makes.
        const float d = __ll2float_rn(index[v + 1] - index[v]);
        const float s = init ? init[v] : x0;
        degf[v] = d;
        score[v] = s;
        gv[v] = __fdiv_rn(s, d);
    }
}

struct OrdCtl {
    GridSync gs;
    int updated[3];  // per sweep, slot sweep % 3
    int sweeps;      // sweeps finished over all launches
    int last_updated;
    int done;
};

struct OrdArgs {
    const int64_t *index;
    const int32_t *nbr;
    const int32_t *order;
    const int32_t *level_off;
    const int32_t *level_long;  // rows of more than kShortRow edges at the head of each level
    int32_t levels, n;
    float *score, *gv;
    const float *degf;
    float damping, eps;
    int32_t sweep_end;  // stop after this many sweeps in total
    OrdCtl *ctl;
};

// The reference's update of row x from its in-order sum: stored only when it
// moves the score by more than eps; returns 1 when stored.
__device__ __forceinline__ int update_row(const OrdArgs &a, float base, int32_t x, float sum) {
    const float nv = __fadd_rn(base, __fmul_rn(a.damping, sum));
    const float old = __ldcg(&a.score[x]);
    if (!(fabsf(__fsub_rn(nv, old)) > a.eps)) return 0;
    __stcg(&a.score[x], nv);
    __stcg(&a.gv[x], __fdiv_rn(nv, a.degf[x]));
    return 1;
}

__global__ void __launch_bounds__(kOrdThreads) pr_ordered_sweeps(OrdArgs a) {
    __shared__ float s_terms[kOrdThreads / 32][kShortRow * 32];
    const int wib = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float base = __fdiv_rn(__fsub_rn(1.0f, a.damping), __int2float_rn(a.n));
    const unsigned long long t_start = globaltimer_ns();
    int s = *(volatile int *)&a.ctl->sweeps;
    for (; s < a.sweep_end; s++) {
        if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->updated[(s + 1) % 3] = 0;
        int local = 0;
        for (int l = 0; l < a.levels; l++) {
            const int lo = a.level_off[l], hi = a.level_off[l + 1];
            // Each level lists its long rows (> kShortRow edges) first.  A long
            // row is summed by one warp (kLongDepth 32-term chunks in flight,
            // summed 32 at a time from shuffles with constant lanes: the add
            // chain is the only wait), one row per warp so that long rows run
            // side by side.  Short rows go 32 to a warp: the warp gathers all
            // their terms at once, coalesced over the rows' concatenated edge
            // ranges, into its shared buffer, and each lane adds its own row's
            // terms in row order.
            const int mid = lo + a.level_long[l];
            for (int i = lo + warp; i < mid; i += nw) {
                const int32_t x = a.order[i];
                const int64_t br = a.index[x], er = a.index[x + 1];
                float sum = 0.0f;
                for (int64_t c0 = br; c0 < er; c0 += 32 * kLongDepth) {
                    float t[kLongDepth];
#pragma unroll
                    for (int j = 0; j < kLongDepth; j++) {
                        const int64_t c = c0 + 32 * j + lane;
                        t[j] = c < er ? __ldcg(&a.gv[a.nbr[c]]) : 0.0f;
                    }
#pragma unroll
                    for (int j = 0; j < kLongDepth; j++) {
                        const int64_t cb = c0 + 32 * j;
                        if (cb >= er) break;
                        if (er - cb >= 32) {
#pragma unroll
                            for (int q = 0; q < 32; q++) sum = __fadd_rn(sum, __shfl_sync(kFull, t[j], q));
                        } else {
                            const int k = (int)(er - cb);
                            for (int q = 0; q < k; q++) sum = __fadd_rn(sum, __shfl_sync(kFull, t[j], q));
                        }
                    }
                }
                int stored = 0;
                if (lane == 0) stored = update_row(a, base, x, sum);
                local += stored;
            }
            for (int g0 = mid + warp * 32; g0 < hi; g0 += nw * 32) {
                const int i = g0 + lane;
                int32_t x = -1;
                int64_t b = 0, e = 0;
                if (i < hi) {
                    x = a.order[i];
                    b = a.index[x];
                    e = a.index[x + 1];
                }
                const int dshort = x >= 0 ? (int)(e - b) : 0;
                int total = 0;
                const int pre = warp_exclusive_scan(dshort, &total);
                for (int k0 = 0; k0 < total; k0 += 32 * kGatherUnroll) {
                    int32_t u[kGatherUnroll];
#pragma unroll
                    for (int j = 0; j < kGatherUnroll; j++) {
                        const int k = k0 + 32 * j + lane;
                        const int kk = min(k, total - 1);
                        // Term kk's row: the last lane whose prefix is <= kk
                        // (every lane takes part in the shuffles).
                        int lo_l = 0;
#pragma unroll
                        for (int st = 16; st > 0; st >>= 1) {
                            const int c = __shfl_sync(kFull, pre, lo_l + st);
                            if (c <= kk) lo_l += st;
                        }
                        const int64_t ob = __shfl_sync(kFull, b, lo_l);
                        const int op = __shfl_sync(kFull, pre, lo_l);
                        u[j] = k < total ? a.nbr[ob + (kk - op)] : -1;
                    }
#pragma unroll
                    for (int j = 0; j < kGatherUnroll; j++) {
                        const int k = k0 + 32 * j + lane;
                        if (k < total) s_terms[wib][k] = __ldcg(&a.gv[u[j]]);
                    }
                }
                __syncwarp();
                if (x >= 0) {
                    float sum = 0.0f;
                    for (int k = pre; k < pre + dshort; k++) sum = __fadd_rn(sum, s_terms[wib][k]);
                    local += update_row(a, base, x, sum);
                }
                __syncwarp();
            }
            if (l == a.levels - 1) {
                const int w = warp_sum(local);
                if (lane == 0 && w) atomicAdd(&a.ctl->updated[s % 3], w);
            }
            if (!grid_barrier(&a.ctl->gs)) return;
        }
        const int u = ld_cg(&a.ctl->updated[s % 3]);
        if (u == 0) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                a.ctl->sweeps = s + 1;
                a.ctl->last_updated = 0;
                a.ctl->done = 1;
            }
            return;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0 && globaltimer_ns() - t_start > c_limits.run_ns)
            atomicExch(&a.ctl->gs.err, (int)HC_ERR_TIMEOUT);
        if (s + 1 == a.sweep_end && blockIdx.x == 0 && threadIdx.x == 0) a.ctl->last_updated = u;
    }
    // Every block leaves here after the same barrier; block 0 records the count.
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->sweeps = s;
}

// Builds the level schedule once per graph: g->pr_ord holds
// order[N] (each level's long rows first) | level_off[levels + 1] |
// level_long[levels] | degf[N], g->pr_ord_levels the count.
hc_status ensure_order(hc_graph *g) {
    if (g->pr_ord_levels >= 0) return HC_OK;
    bool sym = false;
    HC_TRY(ensure_pr_symmetry(g, false, &sym));
    if (!sym)
        return fail(HC_ERR_UNSUPPORTED,
                    "hc_pr_pull_ordered: the graph has an edge without a reverse; the reference's sweep order "
                    "is reproduced for symmetric graphs only");
    const int32_t n = g->N;
    DevBuf cnt, tail;
    HC_TRY(cnt.ensure(sizeof(int32_t) * (size_t)std::max(n, 1)));
    HC_TRY(tail.ensure(sizeof(int32_t)));
    DevBuf order;
    HC_TRY(order.ensure(sizeof(int32_t) * (size_t)std::max(n, 1)));
    HC_CUDA_TRY(cudaMemsetAsync(tail.ptr, 0, sizeof(int32_t), g->stream));
    const int grid = g->sm_count * 8;
    { ord_count_lower<<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(), n, cnt.as<int32_t>(),
                                                   order.as<int32_t>(), tail.as<int32_t>()); count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    std::vector<int32_t> off{0};
    int32_t hi = 0;
    HC_CUDA_TRY(cudaMemcpyAsync(&hi, tail.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    int32_t lo = 0;
    while (hi > lo) {
        off.push_back(hi);
        const int warps_needed = hi - lo;
        const int blocks = std::min(grid, (warps_needed + 7) / 8);
        { ord_expand<<<blocks, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(), order.as<int32_t>(),
                                                    lo, hi, cnt.as<int32_t>(), tail.as<int32_t>()); count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        lo = hi;
        HC_CUDA_TRY(cudaMemcpyAsync(&hi, tail.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    if (lo != n)
        return fail(HC_ERR_INVALID_ARG, "hc_pr_pull_ordered: level schedule placed %d of %d vertices", lo, n);
    const int32_t levels = (int32_t)off.size() - 1;
    // Within a level any order is exact; long rows go first (descending
    // degree, then id), and each level records how many there are.
    std::vector<int32_t> h_order((size_t)n);
    std::vector<int64_t> h_index((size_t)n + 1);
    HC_CUDA_TRY(cudaMemcpyAsync(h_order.data(), order.ptr, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost,
                                g->stream));
    HC_CUDA_TRY(cudaMemcpyAsync(h_index.data(), g->index.ptr, sizeof(int64_t) * ((size_t)n + 1),
                                cudaMemcpyDeviceToHost, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    std::vector<int32_t> nlong((size_t)levels);
    for (int32_t l = 0; l < levels; l++) {
        auto deg = [&](int32_t v) { return h_index[v + 1] - h_index[v]; };
        std::sort(h_order.begin() + off[l], h_order.begin() + off[l + 1], [&](int32_t p, int32_t q) {
            return deg(p) != deg(q) ? deg(p) > deg(q) : p < q;
        });
        int32_t c = 0;
        while (off[l] + c < off[l + 1] && deg(h_order[off[l] + c]) > kShortRow) c++;
        nlong[l] = c;
    }
    const size_t order_b = (sizeof(int32_t) * (size_t)n + 255) / 256 * 256;
    const size_t off_b = (sizeof(int32_t) * (2 * (size_t)levels + 1) + 255) / 256 * 256;
    HC_TRY(g->pr_ord.ensure(order_b + off_b + sizeof(float) * (size_t)n));
    HC_CUDA_TRY(cudaMemcpyAsync(g->pr_ord.ptr, h_order.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice,
                                g->stream));
    HC_CUDA_TRY(cudaMemcpyAsync(g->pr_ord.as<char>() + order_b, off.data(), sizeof(int32_t) * off.size(),
                                cudaMemcpyHostToDevice, g->stream));
    HC_CUDA_TRY(cudaMemcpyAsync(g->pr_ord.as<char>() + order_b + sizeof(int32_t) * off.size(), nlong.data(),
                                sizeof(int32_t) * nlong.size(), cudaMemcpyHostToDevice, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    g->pr_ord_levels = levels;
    return HC_OK;
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_pr_pull_ordered(hc_graph *g, const float *init_scores, float *scores_out,
                                        const hc_pr_opts *opts, hc_pr_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    ReclaimScope reclaim_scope(g, kKeepPrOrd);
    if (!scores_out) return fail(HC_ERR_INVALID_ARG, "hc_pr_pull_ordered: null output");
    hc_pr_opts o{};
    if (opts) o = *opts;
    const float d = o.damping > 0.f ? o.damping : 0.85f;
    const float eps = o.eps_vertex > 0.f ? o.eps_vertex : 5e-8f;
    const int32_t max_sweeps = o.max_iters > 0 ? o.max_iters : 0x7fffffff;
    if (d >= 1.f) return fail(HC_ERR_INVALID_ARG, "hc_pr_pull_ordered: damping must be below 1");
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const int32_t n = g->N;
    if (n == 0) return HC_OK;
    HC_TRY(ensure_order(g));

    const size_t order_b = (sizeof(int32_t) * (size_t)n + 255) / 256 * 256;
    const size_t off_b = (sizeof(int32_t) * (2 * (size_t)g->pr_ord_levels + 1) + 255) / 256 * 256;
    HC_TRY(g->ws_pr.ensure(2 * ((sizeof(float) * (size_t)n + 255) / 256 * 256) + 256));
    HC_TRY(g->ws_ctl.ensure(4096));
    float *score = g->ws_pr.as<float>();
    float *gv = reinterpret_cast<float *>(g->ws_pr.as<char>() + (sizeof(float) * (size_t)n + 255) / 256 * 256);
    float *degf = reinterpret_cast<float *>(g->pr_ord.as<char>() + order_b + off_b);

    const float *init = nullptr;
    if (init_scores) {
        if (is_device_pointer(init_scores)) {
            init = init_scores;
        } else {
            HC_TRY(g->ws_out0.ensure(sizeof(float) * (size_t)n));
            HC_TRY(copy_in(g->ws_out0.ptr, init_scores, sizeof(float) * (size_t)n, g->stream));
            init = g->ws_out0.as<float>();
        }
    }
    OrdCtl *ctl = g->ws_ctl.as<OrdCtl>();
    HC_CUDA_TRY(cudaMemsetAsync(ctl, 0, sizeof(OrdCtl), g->stream));
    HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    { ord_init<<<g->sm_count * 4, 256, 0, g->stream>>>(n, g->index.as<int64_t>(), init, score, gv, degf); count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());

    static int bps = 0;
    if (bps == 0) {
        HC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, pr_ordered_sweeps, kOrdThreads, 0));
        if (bps < 1) return fail(HC_ERR_CUDA, "ordered PageRank kernel cannot be resident");
    }
    // Two blocks per SM: enough warps for the wide levels, and a cheaper
    // barrier for the many narrow ones.
    const int grid = g->sm_count * std::min(bps, 2);
    OrdArgs a{};
    a.index = g->index.as<int64_t>();
    a.nbr = g->nbr.as<int32_t>();
    a.order = g->pr_ord.as<int32_t>();
    a.level_off = reinterpret_cast<const int32_t *>(g->pr_ord.as<char>() + order_b);
    a.level_long = a.level_off + g->pr_ord_levels + 1;
    a.levels = g->pr_ord_levels;
    a.n = n;
    a.score = score;
    a.gv = gv;
    a.degf = degf;
    a.damping = d;
    a.eps = eps;
    a.ctl = ctl;
    OrdCtl h{};
    for (int32_t done = 0; done < max_sweeps;) {
        a.sweep_end = (int32_t)std::min<int64_t>((int64_t)done + kSweepsPerLaunch, max_sweeps);
        void *params[] = {&a};
        count_launch();
        HC_CUDA_TRY(cudaLaunchCooperativeKernel((void *)pr_ordered_sweeps, dim3(grid), dim3(kOrdThreads), params, 0,
                                                g->stream));
        HC_CUDA_TRY(cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        if (h.gs.err) return fail((hc_status)h.gs.err, "hc_pr_pull_ordered: device wait or run limit reached");
        done = h.sweeps;
        if (h.done) break;
    }
    HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    HC_TRY(copy_out(scores_out, score, sizeof(float) * (size_t)n, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (stats) {
        float ms = 0.f;
        HC_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
        stats->iterations = h.sweeps;
        stats->converged = h.done;
        stats->changed = h.done ? 0 : h.last_updated;
        stats->residual_l1 = 0.f;
        stats->bytes_model = (double)h.sweeps * (8.0 * (n + 1) + 4.0 * g->M + 12.0 * n);
        stats->ms = ms;
    }
    return HC_OK;
}
