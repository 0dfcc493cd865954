// Segment profiling of the reference-contract epoch kernels.
//
// The reference's TreeBenchmark (src/benchmarks/benchmark.cuh:87-309,
// src/benchmarks/gpu_benchmark.cuh:201-330) cuts the degree-ordered vertex list
// into segments of about equal edge count (compute_equal_edge_ranges,
// src/graph.cuh:156-201), times one epoch kernel launch restricted to each
// segment (mean of 5 launches, each from the same initial state) and reports
// per segment its degree range, edge count, milliseconds and GTEPS, for 2^d
// segments at each depth d.  These per-segment costs are what a variant
// selector (or the reference's offline scheduler) is fitted to.
//
// hc_profile_segments does that on a resident graph handle: the handle's CSR
// is laid out once in the reference's form (interleaved {int32 v; float w}
// edges, int64 degrees) for the epoch kernels of hc_epoch.cu, and each segment
// is timed with CUDA events on the handle's stream.  SSSP and PageRank start
// every launch from one seeded random vector (as the reference's benchmarks
// do); BFS (a benchmark the reference left unfinished) starts each launch
// from the state before bottom-up level `level` of a BFS from `source`: the
// frontier bitmap of that level and the parents of every vertex reached
// before it.
#include <algorithm>
#include <vector>

#include "hc_graph.cuh"

namespace hc {
namespace {

struct WNode {
    int32_t v;
    float w;
};

__global__ void make_wnodes(const int32_t *nbr, const void *wgt, hc_wtype wt, int64_t m, WNode *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        float w = 1.0f;
        if (wt == HC_W_I32) w = (float)static_cast<const int32_t *>(wgt)[i];
        if (wt == HC_W_F32) w = static_cast<const float *>(wgt)[i];
        out[i] = WNode{nbr[i], w};
    }
}

__global__ void make_degrees(const int64_t *index, int32_t n, int64_t *deg) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        deg[v] = index[v + 1] - index[v];
}

// Seeded uniform (0, 1] floats, counter-based (thread-count independent).
__global__ void seeded_uniform(float *x, int32_t n, uint64_t seed) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        x[v] = (float)((mix64(seed + (uint64_t)v) >> 40) + 1) * (1.0f / 16777216.0f);
}

// BFS state before level `level`: frontier = depth == level; a vertex with
// depth <= level is visited (its parent is any non-negative id).
__global__ void bfs_level_state(const int32_t *depth, int32_t n, int32_t level, uint32_t *frontier, int32_t *parents) {
    const int lane = threadIdx.x & 31;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < ((n + 31) & ~31); v += gridDim.x * blockDim.x) {
        const int32_t d = v < n ? depth[v] : -1;
        const unsigned bits = __ballot_sync(kFull, d == level);
        if (lane == 0) frontier[v >> 5] = bits;
        if (v < n) parents[v] = (d >= 0 && d <= level) ? 0 : -1;
    }
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_equal_edge_ranges(const int64_t *index, int32_t num_nodes, int32_t num_segments,
                                          int32_t chunk_size, int32_t *ranges_out);

extern "C" hc_status hc_profile_segments(hc_graph *g, hc_profile_algo algo, hc_variant variant, int32_t sync_iters,
                                         const int32_t *ranges, int32_t num_segments, int32_t source, int32_t level,
                                         int32_t block_count, int32_t thread_count, int32_t iters,
                                         hc_segment_result *out) {
    clear_error();
    HC_TRY(activate(g));
    if (!ranges || !out || num_segments < 1 || iters < 1 || algo < HC_PROFILE_SSSP || algo > HC_PROFILE_BFS)
        return fail(HC_ERR_INVALID_ARG, "hc_profile_segments: bad arguments");
    const int32_t n = g->N;
    const int64_t m = g->M;
    for (int s = 0; s < num_segments; s++)
        if (ranges[s] < 0 || ranges[s] > ranges[s + 1] || ranges[s + 1] > n)
            return fail(HC_ERR_INVALID_ARG, "hc_profile_segments: segment %d = [%d, %d) outside [0, %d)", s, ranges[s],
                        ranges[s + 1], n);
    if (algo == HC_PROFILE_BFS && (source < 0 || source >= n || level < 0))
        return fail(HC_ERR_INVALID_ARG, "hc_profile_segments: BFS needs a source in [0, N) and a level >= 0");
    std::vector<int64_t> index((size_t)n + 1);
    HC_CUDA_TRY(cudaMemcpyAsync(index.data(), g->index.ptr, sizeof(int64_t) * index.size(), cudaMemcpyDeviceToHost,
                                g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));

    const int grid = g->sm_count * 8;
    DevBuf wn, deg, init, state, work, upd, next, depth;
    HC_TRY(upd.ensure(sizeof(int32_t)));
    const size_t W = ((size_t)n + 31) / 32;
    if (algo != HC_PROFILE_BFS) {
        HC_TRY(wn.ensure(sizeof(WNode) * (size_t)std::max<int64_t>(m, 1)));
        HC_TRY(init.ensure(sizeof(float) * (size_t)n));
        HC_TRY(work.ensure(sizeof(float) * (size_t)n));
        { make_wnodes<<<grid, 256, 0, g->stream>>>(g->nbr.as<int32_t>(), g->wgt.ptr, g->wtype, m, wn.as<WNode>()); count_launch(); }
        { seeded_uniform<<<grid, 256, 0, g->stream>>>(init.as<float>(), n, 1024); count_launch(); }
        if (algo == HC_PROFILE_PR) {
            HC_TRY(deg.ensure(sizeof(int64_t) * (size_t)n));
            { make_degrees<<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), n, deg.as<int64_t>()); count_launch(); }
        }
    } else {
        // The BFS from `source` gives every vertex's level.
        HC_TRY(depth.ensure(sizeof(int32_t) * (size_t)n));
        hc_bfs_opts bo{};
        HC_TRY(hc_bfs(g, &source, 1, depth.as<int32_t>(), nullptr, &bo, nullptr));
        HC_TRY(state.ensure(sizeof(int32_t) * (size_t)n + sizeof(uint32_t) * W));
        HC_TRY(work.ensure(sizeof(int32_t) * (size_t)n));
        HC_TRY(next.ensure(sizeof(uint32_t) * W));
        { bfs_level_state<<<grid, 256, 0, g->stream>>>(depth.as<int32_t>(), n, level,
                                                       reinterpret_cast<uint32_t *>(state.as<int32_t>() + n),
                                                       state.as<int32_t>()); count_launch(); }
    }
    HC_CUDA_TRY(cudaGetLastError());

    cudaEvent_t e0, e1;
    HC_CUDA_TRY(cudaEventCreate(&e0));
    HC_CUDA_TRY(cudaEventCreate(&e1));
    hc_status st = HC_OK;
    for (int s = 0; s < num_segments && st == HC_OK; s++) {
        const int32_t lo = ranges[s], hi = ranges[s + 1];
        hc_segment_result r{};
        r.start_id = lo;
        r.end_id = hi;
        r.num_edges = index[hi] - index[lo];
        r.epoch = algo == HC_PROFILE_BFS ? level : -1;
        if (hi > lo) {
            int64_t dmin = index[lo + 1] - index[lo], dmax = dmin;
            for (int32_t v = lo + 1; v < hi; v++) {
                const int64_t d = index[v + 1] - index[v];
                dmin = std::min(dmin, d);
                dmax = std::max(dmax, d);
            }
            r.avg_degree = (float)r.num_edges / (float)(hi - lo);
            r.min_degree = (float)dmin;
            r.max_degree = (float)dmax;
        }
        double total = 0;
        for (int it = 0; it < iters && st == HC_OK; it++) {
            // Every launch starts from the same state.
            if (algo == HC_PROFILE_BFS) {
                if (cudaMemcpyAsync(work.ptr, state.ptr, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice,
                                    g->stream) != cudaSuccess ||
                    cudaMemsetAsync(next.ptr, 0, sizeof(uint32_t) * W, g->stream) != cudaSuccess)
                    st = fail(HC_ERR_CUDA, "hc_profile_segments: state reset failed");
            } else if (cudaMemcpyAsync(work.ptr, init.ptr, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice,
                                       g->stream) != cudaSuccess) {
                st = fail(HC_ERR_CUDA, "hc_profile_segments: state reset failed");
            }
            if (st == HC_OK && cudaMemsetAsync(upd.ptr, 0, sizeof(int32_t), g->stream) != cudaSuccess)
                st = fail(HC_ERR_CUDA, "hc_profile_segments: counter reset failed");
            if (st != HC_OK) break;
            // The epoch kernels index their rows from `index` at start_id.
            const int64_t *idx = g->index.as<int64_t>() + lo;
            cudaEventRecord(e0, g->stream);
            if (algo == HC_PROFILE_SSSP)
                st = hc_epoch_sssp_pull(idx, wn.ptr, lo, hi, work.as<float>(), upd.as<int32_t>(), variant, block_count,
                                        thread_count, g->stream);
            else if (algo == HC_PROFILE_PR)
                st = hc_epoch_pr_pull(idx, wn.ptr, lo, hi, work.as<float>(), upd.as<int32_t>(), n,
                                      deg.as<int64_t>(), variant, block_count, thread_count, g->stream);
            else if (sync_iters > 0)
                st = hc_epoch_bfs_sync_pull(idx, g->nbr.as<int32_t>(), work.as<int32_t>(), lo, hi,
                                            reinterpret_cast<const uint32_t *>(state.as<int32_t>() + n),
                                            next.as<uint32_t>(), upd.as<int32_t>(), sync_iters, block_count,
                                            thread_count, g->stream);
            else
                st = hc_epoch_bfs_pull(idx, g->nbr.as<int32_t>(), work.as<int32_t>(), lo, hi,
                                       reinterpret_cast<const uint32_t *>(state.as<int32_t>() + n),
                                       next.as<uint32_t>(), upd.as<int32_t>(), variant, block_count, thread_count,
                                       g->stream);
            cudaEventRecord(e1, g->stream);
            if (st != HC_OK) break;
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                st = fail(HC_ERR_CUDA, "hc_profile_segments: %s", cudaGetErrorString(cudaGetLastError()));
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            total += ms;
        }
        r.millis = total / iters;
        // The reference's formula (src/benchmarks/gpu_benchmark.cuh:259): edges / 2 per second.
        r.gteps = r.millis > 0 ? (double)r.num_edges / (r.millis / 1e3) / 1e9 / 2 : 0.0;
        out[s] = r;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}
