// One epoch of the reference's in-place pull kernels, for callers that drive
// their own epoch loop through the epoch-kernel contract of
// src/kernels/kernel_types.cuh:36-63.  Same inputs, outputs and update
// semantics as the reference kernels, written for sm_100a:
//   SSSP  src/kernels/gpu/sssp.cuh:120-281   dist[v] = min(dist[v], dist[u] + w)
//   PR    src/kernels/gpu/pr.cuh:140-318     score[v] = (1-d)/N + d sum score[u]/deg[u]
//   BFS   src/kernels/gpu/bfs.cuh:116-288    bottom-up parent search
// Differences: warp collectives use a full mask (the reference's ALLWARP is
// 0x80000000, src/cuda.cuh:24), the block variants synchronise before the
// shared partials are reused (src/kernels/gpu/sssp.cuh:259-275 races there),
// and the update counter is aggregated per warp before its atomic.
#include <cfloat>

#include "hc_graph.cuh"

namespace hc {
namespace {

struct WNode {
    int32_t v;
    float w;
};

constexpr float kDamp = 0.85f;
constexpr float kPrEps = 5e-8f;

template <class T>
__device__ __forceinline__ T block_reduce_min_or_sum(T v, T *sm, bool is_min) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = is_min ? warp_min(v) : warp_sum(v);
    if (lane == 0) sm[w] = v;
    __syncthreads();
    T r = is_min ? sm[0] : T(0);
    if (threadIdx.x == 0) {
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) r = is_min ? min(r, sm[i]) : r + sm[i];
    }
    __syncthreads();  // partials may be overwritten by the next vertex
    return r;         // valid in thread 0
}

__device__ __forceinline__ void add_count(int32_t *counter, int c) {
    if (blockDim.x & 31) {  // thread-variant blocks need not fill whole warps
        if (c) atomicAdd(counter, c);
        return;
    }
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(counter, c);
}

// ---------------------------------------------------------------- SSSP
__global__ void sssp_epoch_thread(const int64_t *index, const WNode *nb, int32_t s, int32_t e, float *dist,
                                  int32_t *updated) {
    int c = 0;
    const int stride = gridDim.x * blockDim.x;
    const int32_t first = s + blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t span = (e - s + stride - 1) / stride * stride;
    for (int32_t v = first; v < s + span; v += stride) {
        if (v < e) {
            float nd = dist[v];
            const int64_t b = index[v - s], en = index[v - s + 1];
            for (int64_t i = b; i < en; i++) nd = fminf(nd, dist[nb[i].v] + nb[i].w);
            if (nd != dist[v]) {
                dist[v] = nd;
                c++;
            }
        }
    }
    add_count(updated, c);
}

__global__ void sssp_epoch_warp(const int64_t *index, const WNode *nb, int32_t s, int32_t e, float *dist,
                                int32_t *updated) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    int c = 0;
    for (int32_t v = s + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); v < e; v += nw) {
        float nd = dist[v];
        const int64_t b = index[v - s], en = index[v - s + 1];
        for (int64_t i = b + lane; i < en; i += 32) nd = fminf(nd, dist[nb[i].v] + nb[i].w);
        nd = warp_min(nd);
        if (lane == 0 && nd != dist[v]) {
            dist[v] = nd;
            c++;
        }
    }
    if (lane == 0 && c) atomicAdd(updated, c);
}

__global__ void sssp_epoch_block(const int64_t *index, const WNode *nb, int32_t s, int32_t e, float *dist,
                                 int32_t *updated) {
    __shared__ float sm[32];
    int c = 0;
    for (int32_t v = s + blockIdx.x; v < e; v += gridDim.x) {
        float nd = dist[v];
        const int64_t b = index[v - s], en = index[v - s + 1];
        for (int64_t i = b + threadIdx.x; i < en; i += blockDim.x) nd = fminf(nd, dist[nb[i].v] + nb[i].w);
        nd = block_reduce_min_or_sum(nd, sm, true);
        if (threadIdx.x == 0 && nd != dist[v]) {
            dist[v] = nd;
            c++;
        }
    }
    if (threadIdx.x == 0 && c) atomicAdd(updated, c);
}

// ------------------------------------------------------------------ PR
// The thread variant does the reference CPU epoch's fp32 operations one by
// one (src/kernels/cpu/pr.cuh:157-187: divide, add in row order, multiply,
// add; no multiply-add contraction), so a one-thread launch over [0, N)
// sweeps in the single-thread CPU order and reproduces pr_pull_cpu bit for bit.
__global__ void pr_epoch_thread(const int64_t *index, const WNode *nb, int32_t s, int32_t e, float *score,
                                int32_t *updated, int32_t n, const int64_t *deg) {
    int c = 0;
    const float base = __fdiv_rn(__fsub_rn(1.0f, kDamp), __int2float_rn(n));
    const int stride = gridDim.x * blockDim.x;
    const int32_t span = (e - s + stride - 1) / stride * stride;
    for (int32_t v = s + blockIdx.x * blockDim.x + threadIdx.x; v < s + span; v += stride) {
        if (v < e) {
            float t = 0.f;
            const int64_t b = index[v - s], en = index[v - s + 1];
            for (int64_t i = b; i < en; i++) {
                const int32_t u = nb[i].v;
                t = __fadd_rn(t, __fdiv_rn(score[u], __ll2float_rn(deg[u])));
            }
            const float ns = __fadd_rn(base, __fmul_rn(kDamp, t));
            if (fabsf(__fsub_rn(ns, score[v])) > kPrEps) {
                score[v] = ns;
                c++;
            }
        }
    }
    add_count(updated, c);
}

__global__ void pr_epoch_warp(const int64_t *index, const WNode *nb, int32_t s, int32_t e, float *score,
                              int32_t *updated, int32_t n, const int64_t *deg) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float base = (1.0f - kDamp) / n;
    int c = 0;
    for (int32_t v = s + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); v < e; v += nw) {
        float t = 0.f;
        const int64_t b = index[v - s], en = index[v - s + 1];
        for (int64_t i = b + lane; i < en; i += 32) {
            const int32_t u = nb[i].v;
            t += score[u] / (float)deg[u];
        }
        t = warp_sum(t);
        const float ns = base + kDamp * t;
        if (lane == 0 && fabsf(ns - score[v]) > kPrEps) {
            score[v] = ns;
            c++;
        }
    }
    if (lane == 0 && c) atomicAdd(updated, c);
}

__global__ void pr_epoch_block(const int64_t *index, const WNode *nb, int32_t s, int32_t e, float *score,
                               int32_t *updated, int32_t n, const int64_t *deg) {
    __shared__ float sm[32];
    const float base = (1.0f - kDamp) / n;
    int c = 0;
    for (int32_t v = s + blockIdx.x; v < e; v += gridDim.x) {
        float t = 0.f;
        const int64_t b = index[v - s], en = index[v - s + 1];
        for (int64_t i = b + threadIdx.x; i < en; i += blockDim.x) {
            const int32_t u = nb[i].v;
            t += score[u] / (float)deg[u];
        }
        t = block_reduce_min_or_sum(t, sm, false);
        if (threadIdx.x == 0) {
            const float ns = base + kDamp * t;
            if (fabsf(ns - score[v]) > kPrEps) {
                score[v] = ns;
                c++;
            }
        }
    }
    if (threadIdx.x == 0 && c) atomicAdd(updated, c);
}

// ----------------------------------------------------------------- BFS
__device__ __forceinline__ bool in_frontier(const uint32_t *f, int32_t u) { return (f[u >> 5] >> (u & 31)) & 1u; }

__global__ void bfs_epoch_thread(const int64_t *index, const int32_t *nbr, int32_t *parents, int32_t s, int32_t e,
                                 const uint32_t *frontier, uint32_t *next, int32_t *count) {
    int c = 0;
    const int stride = gridDim.x * blockDim.x;
    const int32_t span = (e - s + stride - 1) / stride * stride;
    for (int32_t v = s + blockIdx.x * blockDim.x + threadIdx.x; v < s + span; v += stride) {
        if (v < e && parents[v] == -1) {
            const int64_t b = index[v - s], en = index[v - s + 1];
            for (int64_t i = b; i < en; i++) {
                const int32_t u = nbr[i];
                if (in_frontier(frontier, u)) {
                    parents[v] = u;
                    atomicOr(next + (v >> 5), 1u << (v & 31));
                    c++;
                    break;
                }
            }
        }
    }
    add_count(count, c);
}

__global__ void bfs_epoch_warp(const int64_t *index, const int32_t *nbr, int32_t *parents, int32_t s, int32_t e,
                               const uint32_t *frontier, uint32_t *next, int32_t *count) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    int c = 0;
    for (int32_t v = s + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); v < e; v += nw) {
        if (parents[v] != -1) continue;
        const int64_t b = index[v - s], en = index[v - s + 1];
        for (int64_t i0 = b; i0 < en; i0 += 32) {
            const int64_t i = i0 + lane;
            const bool hit = i < en && in_frontier(frontier, nbr[i]);
            const unsigned bal = __ballot_sync(kFull, hit);
            if (bal) {
                const int32_t p = __shfl_sync(kFull, i < en ? nbr[i] : 0, __ffs(bal) - 1);
                if (lane == 0) {
                    parents[v] = p;
                    atomicOr(next + (v >> 5), 1u << (v & 31));
                    c++;
                }
                break;
            }
        }
    }
    if (lane == 0 && c) atomicAdd(count, c);
}

// The sync-warp variant (src/kernels/gpu/bfs.cuh:234-288): the warp probes
// sync_iters 32-edge chunks of the row before it votes, trading wasted probes
// for fewer votes.  The parent taken is the first frontier neighbour in row
// order among the probed chunks.
__global__ void bfs_epoch_sync_warp(const int64_t *index, const int32_t *nbr, int32_t *parents, int32_t s, int32_t e,
                                    const uint32_t *frontier, uint32_t *next, int32_t *count, int sync_iters) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    int c = 0;
    for (int32_t v = s + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); v < e; v += nw) {
        if (parents[v] != -1) continue;
        const int64_t b = index[v - s], en = index[v - s + 1];
        const int64_t chunks = (en - b + 31) / 32;
        for (int64_t c0 = 0; c0 < chunks; c0 += sync_iters) {
            int first = 0x7fffffff;  // (chunk within the group) * 32 + lane of this lane's first hit
            int32_t hit = 0;
            for (int k = 0; k < sync_iters && first == 0x7fffffff; k++) {
                const int64_t i = b + (c0 + k) * 32 + lane;
                if (i < en) {
                    const int32_t u = nbr[i];
                    if (in_frontier(frontier, u)) {
                        first = k * 32 + lane;
                        hit = u;
                    }
                }
            }
            const int best = warp_min(first);
            if (best != 0x7fffffff) {
                const int32_t p = __shfl_sync(kFull, hit, best & 31);
                if (lane == 0) {
                    parents[v] = p;
                    atomicOr(next + (v >> 5), 1u << (v & 31));
                    c++;
                }
                break;
            }
        }
    }
    if (lane == 0 && c) atomicAdd(count, c);
}

hc_status check_shape(int32_t blocks, int32_t threads, hc_variant v) {
    if (blocks < 1 || threads < 1 || threads > 1024)
        return fail(HC_ERR_INVALID_ARG, "epoch launch shape %d x %d is invalid", blocks, threads);
    // Same rule as the reference drivers (src/kernels/gpu/sssp.cuh:47-49).
    if (v != HC_VARIANT_THREAD && threads % 32 != 0)
        return fail(HC_ERR_INVALID_ARG, "thread count must be divisible by 32");
    return HC_OK;
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" {

hc_status hc_epoch_sssp_pull(const int64_t *index, const void *wnodes, int32_t start_id, int32_t end_id, float *dist,
                             int32_t *updated, hc_variant variant, int32_t block_count, int32_t thread_count,
                             void *stream) {
    clear_error();
    if (!index || !dist || !updated || start_id > end_id || start_id < 0)
        return fail(HC_ERR_INVALID_ARG, "hc_epoch_sssp_pull: bad arguments");
    HC_TRY(check_shape(block_count, thread_count, variant));
    if (start_id == end_id) return HC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const WNode *nb = (const WNode *)wnodes;
    switch (variant) {
        case HC_VARIANT_THREAD:
            { sssp_epoch_thread<<<block_count, thread_count, 0, s>>>(index, nb, start_id, end_id, dist, updated); ::hc::count_launch(); }
            break;
        case HC_VARIANT_BLOCK:
            { sssp_epoch_block<<<block_count, thread_count, 0, s>>>(index, nb, start_id, end_id, dist, updated); ::hc::count_launch(); }
            break;
        default:
            { sssp_epoch_warp<<<block_count, thread_count, 0, s>>>(index, nb, start_id, end_id, dist, updated); ::hc::count_launch(); }
            break;
    }
    HC_CUDA_TRY(cudaGetLastError());
    return HC_OK;
}

hc_status hc_epoch_pr_pull(const int64_t *index, const void *wnodes, int32_t start_id, int32_t end_id, float *score,
                           int32_t *updated, int32_t num_nodes, const int64_t *degrees, hc_variant variant,
                           int32_t block_count, int32_t thread_count, void *stream) {
    clear_error();
    if (!index || !score || !updated || !degrees || start_id > end_id || start_id < 0 || num_nodes < 1)
        return fail(HC_ERR_INVALID_ARG, "hc_epoch_pr_pull: bad arguments");
    HC_TRY(check_shape(block_count, thread_count, variant));
    if (start_id == end_id) return HC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const WNode *nb = (const WNode *)wnodes;
    switch (variant) {
        case HC_VARIANT_THREAD:
            { pr_epoch_thread<<<block_count, thread_count, 0, s>>>(index, nb, start_id, end_id, score, updated, num_nodes,
                                                                 degrees); ::hc::count_launch(); }
            break;
        case HC_VARIANT_BLOCK:
            { pr_epoch_block<<<block_count, thread_count, 0, s>>>(index, nb, start_id, end_id, score, updated, num_nodes,
                                                                degrees); ::hc::count_launch(); }
            break;
        default:
            { pr_epoch_warp<<<block_count, thread_count, 0, s>>>(index, nb, start_id, end_id, score, updated, num_nodes,
                                                               degrees); ::hc::count_launch(); }
            break;
    }
    HC_CUDA_TRY(cudaGetLastError());
    return HC_OK;
}

hc_status hc_epoch_bfs_pull(const int64_t *index, const int32_t *neighbors, int32_t *parents, int32_t start_id,
                            int32_t end_id, const uint32_t *frontier, uint32_t *next_frontier, int32_t *num_nodes,
                            hc_variant variant, int32_t block_count, int32_t thread_count, void *stream) {
    clear_error();
    if (!index || !parents || !frontier || !next_frontier || !num_nodes || start_id > end_id || start_id < 0)
        return fail(HC_ERR_INVALID_ARG, "hc_epoch_bfs_pull: bad arguments");
    HC_TRY(check_shape(block_count, thread_count, variant));
    if (start_id == end_id) return HC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (variant == HC_VARIANT_THREAD)
        { bfs_epoch_thread<<<block_count, thread_count, 0, s>>>(index, neighbors, parents, start_id, end_id, frontier,
                                                              next_frontier, num_nodes); ::hc::count_launch(); }
    else
        { bfs_epoch_warp<<<block_count, thread_count, 0, s>>>(index, neighbors, parents, start_id, end_id, frontier,
                                                            next_frontier, num_nodes); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    return HC_OK;
}

hc_status hc_epoch_bfs_sync_pull(const int64_t *index, const int32_t *neighbors, int32_t *parents, int32_t start_id,
                                 int32_t end_id, const uint32_t *frontier, uint32_t *next_frontier, int32_t *num_nodes,
                                 int32_t sync_iters, int32_t block_count, int32_t thread_count, void *stream) {
    clear_error();
    if (!index || !parents || !frontier || !next_frontier || !num_nodes || start_id > end_id || start_id < 0 ||
        sync_iters < 1)
        return fail(HC_ERR_INVALID_ARG, "hc_epoch_bfs_sync_pull: bad arguments");
    HC_TRY(check_shape(block_count, thread_count, HC_VARIANT_WARP));
    if (start_id == end_id) return HC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    { bfs_epoch_sync_warp<<<block_count, thread_count, 0, s>>>(index, neighbors, parents, start_id, end_id, frontier,
                                                             next_frontier, num_nodes, sync_iters); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    return HC_OK;
}

}  // extern "C"
