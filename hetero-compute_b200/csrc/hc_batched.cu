// Batched multi-source BFS and SSSP.
//
// The reference runs sources one after another, each a full driver call
// (src/benchmarks/gpu_benchmark.cuh:577-586).  Here a group of sources shares
// every sweep over the CSR:
//
// BFS (bit-sliced frontiers, after Then et al., "The more the merrier:
// efficient multi-source graph traversal", VLDB 2014): per vertex, K64 64-bit
// words of `seen`, `front` and `next` bits, one bit per source, vertex-major so
// a neighbour's frontier is one contiguous 8*K64-byte gather.  A level is a
// pull over every vertex still missing some source: next[v] = OR_u front[u]
// & ~seen[v], skipping neighbours whose frontier is empty (1-bit activity
// map).  K64 lanes of a warp own one vertex.
//
// SSSP: distances vertex-major dist[v][32] (one lane per source, 128-byte rows),
// an activity mask per vertex (bit s = distance for source s dropped last
// epoch) and a queue of active vertices.  An epoch relaxes every edge out of
// the queue for all sources whose bit is set, int32 atomicMin per lane.  Rows
// longer than kLongRow are cut into chunks processed by a second launch.
#include <algorithm>
#include <vector>

#include "hc_graph.cuh"

namespace hc {
namespace {

// ------------------------------------------------------------------- BFS

template <int K64>
__global__ void msbfs_init(int32_t n, int nsrc, const int32_t *src, uint64_t *seen, uint64_t *front,
                           uint32_t *act, int W) {
    const size_t total = (size_t)n * K64;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        seen[i] = 0;
        front[i] = 0;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < W; i += gridDim.x * blockDim.x) act[i] = 0;
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

// One pull level.  Lane j of a K64-lane group owns word j of vertex v.
template <int K64>
__global__ void __launch_bounds__(256) msbfs_level(const int64_t *index, const int32_t *nbr, int32_t n_active,
                                                   int nsrc, const uint64_t *seen_in, uint64_t *seen_out,
                                                   const uint64_t *front, uint64_t *next, const uint32_t *act,
                                                   uint32_t *act_next, int32_t *depth, int64_t n, int level,
                                                   unsigned long long *found) {
    constexpr int G = 32 / K64;  // vertices per warp
    const int lane = threadIdx.x & 31;
    const int sub = lane % K64, grp = lane / K64;
    const unsigned gmask = (K64 == 32 ? 0xffffffffu : ((1u << K64) - 1u)) << (grp * K64);
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    // Valid-source mask of this lane's word.
    const int bits_here = min(64, max(0, nsrc - sub * 64));
    const uint64_t fm = bits_here >= 64 ? ~0ull : ((1ull << bits_here) - 1ull);
    unsigned long long my_found = 0;
    for (int32_t vb = gwarp * G; vb < n_active; vb += nwarps * G) {
        const int32_t v = vb + grp;
        const bool valid = v < n_active;
        uint64_t s = valid ? seen_in[(size_t)v * K64 + sub] : fm;
        uint64_t acc = 0;
        // Vertex done for every source: skip its row (group-uniform).
        const bool need = __any_sync(kFull, valid && (s & fm) != fm);
        if (need) {
            const bool mine = __any_sync(gmask, (s & fm) != fm) && valid;
            int64_t b = 0, e = 0;
            if (mine) {
                b = index[v];
                e = index[v + 1];
            }
            for (int64_t i = b; i < e; i++) {
                const int32_t u = nbr[i];
                if ((act[u >> 5] >> (u & 31)) & 1u) acc |= front[(size_t)u * K64 + sub];
            }
        }
        const uint64_t nw = acc & ~s & fm;
        if (valid) {
            next[(size_t)v * K64 + sub] = nw;
            seen_out[(size_t)v * K64 + sub] = s | nw;
            if (nw && depth) {
                uint64_t x = nw;
                while (x) {
                    const int b = __ffsll((long long)x) - 1;
                    x &= x - 1;
                    depth[(size_t)(sub * 64 + b) * n + v] = level + 1;
                }
            }
        }
        const bool any_new = __any_sync(gmask, nw != 0);
        if (valid && sub == 0 && any_new) {
            atomicOr(act_next + (v >> 5), 1u << (v & 31));
            my_found++;
        }
    }
    my_found = warp_sum(my_found);
    if (lane == 0 && my_found) atomicAdd(found, my_found);
}

// ------------------------------------------------------------------ SSSP

constexpr int kLongRow = 2048;

__global__ void mssp_init(int32_t n, int32_t *dist, uint32_t *act0, uint32_t *act1) {
    const size_t total = (size_t)n * 32;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        dist[i] = kInfDist;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        act0[i] = 0;
        act1[i] = 0;
    }
}

__global__ void mssp_seed(int nsrc, const int32_t *src, int32_t *dist, uint32_t *act, int32_t *queue, int *qlen) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int q = 0;
        for (int s = 0; s < nsrc; s++) {
            const int32_t v = src[s];
            dist[(size_t)v * 32 + s] = 0;
            if (act[v] == 0) queue[q++] = v;
            act[v] |= 1u << s;
        }
        *qlen = q;
    }
}

// Relax 32 consecutive edges [e0, e1) of row u for the sources in `m`.
__device__ __forceinline__ void mssp_relax_range(const int32_t *nbr, const int32_t *w, int32_t *dist, uint32_t m,
                                                 int32_t du, int64_t e0, int64_t e1, uint32_t *act_next,
                                                 int32_t *qnext, int *qlen, unsigned long long &relaxed) {
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
        for (int j = 0; j < cnt; j++) {
            const int32_t v = __shfl_sync(kFull, vv, j);
            const int32_t wt = __shfl_sync(kFull, ww, j);
            bool imp = false;
            if (on) {
                const int32_t nd = du + wt;
                int32_t *dp = dist + (size_t)v * 32 + lane;
                if (nd < __ldcg(dp)) imp = nd < atomicMin(dp, nd);
            }
            const unsigned bal = __ballot_sync(kFull, imp);
            if (bal && lane == 0) {
                const uint32_t old = atomicOr(act_next + v, bal);
                if (old == 0) qnext[atomicAdd(qlen, 1)] = v;
            }
        }
        relaxed += (unsigned long long)cnt * __popc(m);
    }
}

__global__ void __launch_bounds__(256) mssp_epoch(const int64_t *index, const int32_t *nbr, const int32_t *w,
                                                  int32_t *dist, const int32_t *qcur, int nq, const uint32_t *act_cur,
                                                  uint32_t *act_next, int32_t *qnext, int *qnext_len, int2 *tasks,
                                                  int *ntasks, unsigned long long *relaxed) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long rel = 0;
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
        const int32_t du = __ldcg(dist + (size_t)u * 32 + lane);
        mssp_relax_range(nbr, w, dist, m, du, b, e, act_next, qnext, qnext_len, rel);
    }
    rel = warp_sum(rel);
    if (lane == 0 && rel) atomicAdd(relaxed, rel);
}

__global__ void __launch_bounds__(256) mssp_tasks(const int64_t *index, const int32_t *nbr, const int32_t *w,
                                                  int32_t *dist, const int2 *tasks, const int *ntasks,
                                                  const uint32_t *act_cur, uint32_t *act_next, int32_t *qnext,
                                                  int *qnext_len, unsigned long long *relaxed) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nt = *ntasks;
    unsigned long long rel = 0;
    for (int t = gwarp; t < nt; t += nwarps) {
        const int2 tk = tasks[t];
        const int32_t u = tk.x;
        const uint32_t m = act_cur[u];
        const int64_t rb = index[u], re = index[u + 1];
        const int64_t b = rb + (int64_t)tk.y * kLongRow;
        const int64_t e = (re < b + kLongRow) ? re : b + kLongRow;
        const int32_t du = __ldcg(dist + (size_t)u * 32 + lane);
        mssp_relax_range(nbr, w, dist, m, du, b, e, act_next, qnext, qnext_len, rel);
    }
    rel = warp_sum(rel);
    if (lane == 0 && rel) atomicAdd(relaxed, rel);
}

__global__ void mssp_clear(const int32_t *q, int nq, uint32_t *act) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) act[q[i]] = 0;
}

// dist[v][32] -> out[s][v] for the group's sources, 32x32 tiles through shared memory.
__global__ void mssp_transpose(const int32_t *dist, int32_t n, int nsrc, int32_t *out) {
    __shared__ int32_t tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int64_t vb = (int64_t)blockIdx.x * 32; vb < n; vb += (int64_t)gridDim.x * 32) {
        for (int r = ty; r < 32; r += 8) {
            const int64_t v = vb + r;
            tile[r][tx] = v < n ? dist[(size_t)v * 32 + tx] : 0;
        }
        __syncthreads();
        for (int s = ty; s < nsrc; s += 8) {
            const int64_t v = vb + tx;
            if (v < n) out[(size_t)s * n + v] = tile[tx][s];
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace hc

using namespace hc;

namespace {

template <int K64>
hc_status run_msbfs(hc_graph *g, const int32_t *d_src, int nsrc, int32_t *depth, const hc_batch_opts &o,
                    int *levels_out, double *bytes) {
    const int64_t n = g->N;
    const int W = (int)((n + 31) / 32);
    const size_t nk = (size_t)n * K64;
    HC_TRY(g->ws_batch.ensure(nk * 8 * 4 + (size_t)W * 4 * 2 + 4096));
    char *p = g->ws_batch.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    uint64_t *seen[2] = {(uint64_t *)take(nk * 8), (uint64_t *)take(nk * 8)};
    uint64_t *fr[2] = {(uint64_t *)take(nk * 8), (uint64_t *)take(nk * 8)};
    uint32_t *act[2] = {(uint32_t *)take((size_t)W * 4), (uint32_t *)take((size_t)W * 4)};
    unsigned long long *found = (unsigned long long *)take(64);
    const int grid = g->sm_count * 8;
    { msbfs_init<K64><<<grid, 256, 0, g->stream>>>(g->N, nsrc, d_src, seen[0], fr[0], act[0], W); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaMemsetAsync(act[1], 0, (size_t)W * 4, g->stream));
    if (depth) HC_CUDA_TRY(cudaMemsetAsync(depth, 0xff, sizeof(int32_t) * (size_t)nsrc * n, g->stream));
    { msbfs_seed<K64><<<(nsrc + 255) / 256, 256, 0, g->stream>>>(nsrc, d_src, seen[0], fr[0], act[0], depth, n); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    const int max_levels = o.max_epochs > 0 ? o.max_epochs : g->N + 1;
    int level = 0;
    double b = 0;
    for (; level < max_levels; level++) {
        const int c = level & 1;
        HC_CUDA_TRY(cudaMemsetAsync(found, 0, 8, g->stream));
        HC_CUDA_TRY(cudaMemsetAsync(act[c ^ 1], 0, (size_t)W * 4, g->stream));
        { msbfs_level<K64><<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(), g->n_active, nsrc,
                                                      seen[c], seen[c ^ 1], fr[c], fr[c ^ 1], act[c], act[c ^ 1],
                                                      depth, n, level, found); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        unsigned long long h = 0;
        HC_CUDA_TRY(cudaMemcpyAsync(&h, found, 8, cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        // Offsets + neighbours once per level, plus seen/next words per vertex.
        b += 8.0 * (n + 1) + 4.0 * g->M + 3.0 * 8.0 * K64 * (double)g->n_active;
        if (h == 0) {
            level++;
            break;
        }
    }
    *levels_out = level;
    *bytes = b;
    return HC_OK;
}

}  // namespace

extern "C" hc_status hc_bfs_batched(hc_graph *g, const int32_t *sources, int32_t num_sources, int32_t *depth_out,
                                    const hc_batch_opts *opts, hc_batch_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    if (!sources || num_sources < 1) return fail(HC_ERR_INVALID_ARG, "hc_bfs_batched: bad source list");
    hc_batch_opts o{};
    if (opts) o = *opts;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    std::vector<int32_t> src(num_sources);
    HC_CUDA_TRY(cudaMemcpy(src.data(), sources, sizeof(int32_t) * num_sources, cudaMemcpyDefault));
    for (int32_t s : src)
        if (s < 0 || s >= g->N) return fail(HC_ERR_INVALID_ARG, "hc_bfs_batched: source %d out of range", s);
    const int group = o.group > 0 ? std::min(o.group, 512) : 512;
    const int64_t n = g->N;
    const bool dev_out = is_device_pointer(depth_out);
    int32_t *d_src = nullptr;
    HC_CUDA_TRY(cudaMalloc(&d_src, sizeof(int32_t) * num_sources));
    struct Free {
        int32_t *p;
        ~Free() { cudaFree(p); }
    } fr{d_src};
    HC_CUDA_TRY(cudaMemcpy(d_src, src.data(), sizeof(int32_t) * num_sources, cudaMemcpyHostToDevice));
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
        if (k64 <= 1) HC_TRY(run_msbfs<1>(g, d_src + s0, k, dep, o, &lv, &b));
        else if (k64 <= 2) HC_TRY(run_msbfs<2>(g, d_src + s0, k, dep, o, &lv, &b));
        else if (k64 <= 4) HC_TRY(run_msbfs<4>(g, d_src + s0, k, dep, o, &lv, &b));
        else HC_TRY(run_msbfs<8>(g, d_src + s0, k, dep, o, &lv, &b));
        if (depth_out && !dev_out) HC_TRY(copy_out(depth_out + (size_t)s0 * n, dep, sizeof(int32_t) * (size_t)k * n, g->stream));
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

extern "C" hc_status hc_sssp_batched(hc_graph *g, const int32_t *sources, int32_t num_sources, int32_t *dist_out,
                                     const hc_batch_opts *opts, hc_batch_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    if (!sources || num_sources < 1) return fail(HC_ERR_INVALID_ARG, "hc_sssp_batched: bad source list");
    if (g->wtype != HC_W_I32) return fail(HC_ERR_UNSUPPORTED, "hc_sssp_batched: graph needs int32 edge weights");
    hc_batch_opts o{};
    if (opts) o = *opts;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    std::vector<int32_t> src(num_sources);
    HC_CUDA_TRY(cudaMemcpy(src.data(), sources, sizeof(int32_t) * num_sources, cudaMemcpyDefault));
    for (int32_t s : src)
        if (s < 0 || s >= g->N) return fail(HC_ERR_INVALID_ARG, "hc_sssp_batched: source %d out of range", s);
    const int64_t n = g->N;
    const int64_t max_tasks = 2 * (g->M / kLongRow) + n / kLongRow + 64;
    HC_TRY(g->ws_batch.ensure((size_t)n * 32 * 4 + (size_t)n * 4 * 4 + sizeof(int2) * max_tasks + 8192));
    char *p = g->ws_batch.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    int32_t *dist = (int32_t *)take((size_t)n * 32 * 4);
    uint32_t *act[2] = {(uint32_t *)take((size_t)n * 4), (uint32_t *)take((size_t)n * 4)};
    int32_t *q[2] = {(int32_t *)take((size_t)n * 4), (int32_t *)take((size_t)n * 4)};
    int2 *tasks = (int2 *)take(sizeof(int2) * max_tasks);
    int *ctr = (int *)take(256);  // [0],[1] queue lengths, [2] tasks
    unsigned long long *relaxed = (unsigned long long *)take(64);
    int32_t *d_src = (int32_t *)take(sizeof(int32_t) * 32);
    const bool dev_out = is_device_pointer(dist_out);
    if (dist_out && !dev_out) HC_TRY(g->ws_out0.ensure(sizeof(int32_t) * (size_t)32 * n));
    const int grid = g->sm_count * 8;
    const int max_epochs = o.max_epochs > 0 ? o.max_epochs : 0x7fffffff;
    HC_CUDA_TRY(cudaMemsetAsync(relaxed, 0, 8, g->stream));
    HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    int epochs_max = 0, groups = 0;
    for (int s0 = 0; s0 < num_sources; s0 += 32, groups++) {
        const int k = std::min(32, num_sources - s0);
        HC_CUDA_TRY(cudaMemcpyAsync(d_src, src.data() + s0, sizeof(int32_t) * k, cudaMemcpyHostToDevice, g->stream));
        { mssp_init<<<grid, 256, 0, g->stream>>>(g->N, dist, act[0], act[1]); ::hc::count_launch(); }
        { mssp_seed<<<1, 32, 0, g->stream>>>(k, d_src, dist, act[0], q[0], &ctr[0]); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        int nq = 0;
        HC_CUDA_TRY(cudaMemcpyAsync(&nq, &ctr[0], 4, cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        int ep = 0;
        for (; nq > 0; ep++) {
            if (ep >= max_epochs) return fail(HC_ERR_NOT_CONVERGED, "hc_sssp_batched: epoch cap reached");
            const int c = ep & 1;
            HC_CUDA_TRY(cudaMemsetAsync(&ctr[c ^ 1], 0, 4, g->stream));
            HC_CUDA_TRY(cudaMemsetAsync(&ctr[2], 0, 4, g->stream));
            { mssp_epoch<<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(), g->wgt.as<int32_t>(),
                                                    dist, q[c], nq, act[c], act[c ^ 1], q[c ^ 1], &ctr[c ^ 1], tasks,
                                                    &ctr[2], relaxed); ::hc::count_launch(); }
            { mssp_tasks<<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(), g->wgt.as<int32_t>(),
                                                    dist, tasks, &ctr[2], act[c], act[c ^ 1], q[c ^ 1], &ctr[c ^ 1],
                                                    relaxed); ::hc::count_launch(); }
            { mssp_clear<<<(nq + 255) / 256, 256, 0, g->stream>>>(q[c], nq, act[c]); ::hc::count_launch(); }
            HC_CUDA_TRY(cudaGetLastError());
            HC_CUDA_TRY(cudaMemcpyAsync(&nq, &ctr[c ^ 1], 4, cudaMemcpyDeviceToHost, g->stream));
            HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        }
        epochs_max = std::max(epochs_max, ep);
        if (dist_out) {
            int32_t *dst = dev_out ? dist_out + (size_t)s0 * n : g->ws_out0.as<int32_t>();
            { mssp_transpose<<<grid, 256, 0, g->stream>>>(dist, g->N, k, dst); ::hc::count_launch(); }
            HC_CUDA_TRY(cudaGetLastError());
            if (!dev_out) HC_TRY(copy_out(dist_out + (size_t)s0 * n, dst, sizeof(int32_t) * (size_t)k * n, g->stream));
        }
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
        // 8 B (neighbour + weight) per edge visit of a row, amortised over the
        // group's lanes, plus a 128-byte distance row per relaxed edge visit.
        stats->bytes_model = (double)rel / 32.0 * (8.0 + 128.0);
    }
    return HC_OK;
}
