// Batched multi-source SSSP.
//
// The reference runs sources one after another (src/benchmarks/gpu_benchmark.cuh:577-586),
// each a full Bellman-Ford pull (src/kernels/gpu/sssp.cuh:42-100).  Here a group
// of K = 32 * SPL sources shares every sweep: distances are vertex-major,
// dist[v][K], lane l of a warp owns sources l*SPL .. l*SPL+SPL-1 and reads them
// with one SPL-wide vector load, so the distances of a vertex for the whole
// group are one contiguous 4K-byte row.  An activity mask per vertex (bit l =
// one of lane l's distances dropped last epoch) and a queue of active vertices
// drive the epochs: every edge out of the queue is relaxed for the active
// lanes, a warp keeping four edges in flight (row loads, then atomicMins, then
// the activity updates of the four targets).  Rows longer than kLongRow are
// cut into chunks processed by a second launch.  Wider groups amortise the row
// reads over more sources; the frontiers of Kronecker sources overlap, so the
// union frontier grows more slowly than the group.
#include <algorithm>
#include <vector>

#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr int kLongRow = 2048;

template <int SPL>
__device__ __forceinline__ void load_row(const int32_t *p, int32_t (&d)[SPL]) {
    if constexpr (SPL == 1) {
        d[0] = __ldcg(p);
    } else if constexpr (SPL == 2) {
        const int2 x = __ldcg(reinterpret_cast<const int2 *>(p));
        d[0] = x.x;
        d[1] = x.y;
    } else {
        const int4 x = __ldcg(reinterpret_cast<const int4 *>(p));
        d[0] = x.x;
        d[1] = x.y;
        d[2] = x.z;
        d[3] = x.w;
    }
}

template <int SPL>
__global__ void mssp_init(int32_t n, int32_t *dist, uint32_t *act0, uint32_t *act1) {
    const size_t total = (size_t)n * 32 * SPL;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        dist[i] = kInfDist;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        act0[i] = 0;
        act1[i] = 0;
    }
}

template <int SPL>
__global__ void mssp_seed(int nsrc, const int32_t *src, int32_t *dist, uint32_t *act, int32_t *queue, int *qlen) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int q = 0;
        for (int s = 0; s < nsrc; s++) {
            const int32_t v = src[s];
            dist[(size_t)v * 32 * SPL + s] = 0;
            if (act[v] == 0) queue[q++] = v;
            act[v] |= 1u << (s / SPL);
        }
        *qlen = q;
    }
}

// Relax edges [e0, e1) of row u for the active lanes in `m`; du = this lane's
// distances of u.
template <int SPL>
__device__ __forceinline__ void relax_range(const int32_t *nbr, const int32_t *w, int32_t *dist, uint32_t m,
                                            const int32_t (&du)[SPL], int64_t e0, int64_t e1, uint32_t *act_next,
                                            int32_t *qnext, int *qlen, unsigned long long &relaxed) {
    constexpr int K = 32 * SPL;
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
        for (int j0 = 0; j0 < cnt; j0 += 4) {
            int32_t v[4], wt[4], d[4][SPL];
            bool ok[4], imp[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int idx = j0 + k;
                v[k] = __shfl_sync(kFull, vv, idx & 31);
                wt[k] = __shfl_sync(kFull, ww, idx & 31);
                ok[k] = on && idx < cnt;
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (ok[k]) {
                    load_row<SPL>(dist + (size_t)v[k] * K + lane * SPL, d[k]);
                } else {
#pragma unroll
                    for (int s = 0; s < SPL; s++) d[k][s] = kInfDist;
                }
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                imp[k] = false;
#pragma unroll
                for (int s = 0; s < SPL; s++) {
                    const int32_t nd = du[s] == kInfDist ? kInfDist : du[s] + wt[k];
                    if (ok[k] && nd < d[k][s] && nd < atomicMin(dist + (size_t)v[k] * K + lane * SPL + s, nd))
                        imp[k] = true;
                }
            }
            unsigned bal[4];
#pragma unroll
            for (int k = 0; k < 4; k++) bal[k] = __ballot_sync(kFull, imp[k]);
            const unsigned mybal = lane == 0 ? bal[0] : lane == 1 ? bal[1] : lane == 2 ? bal[2] : lane == 3 ? bal[3] : 0u;
            const int32_t myv = lane == 0 ? v[0] : lane == 1 ? v[1] : lane == 2 ? v[2] : v[3];
            bool app = false;
            if (mybal) app = atomicOr(act_next + myv, mybal) == 0u;
            const unsigned ap = __ballot_sync(kFull, app);
            if (ap) {
                int base_q = 0;
                const int leader = __ffs(ap) - 1;
                if (lane == leader) base_q = atomicAdd(qlen, __popc(ap));
                base_q = __shfl_sync(kFull, base_q, leader);
                if (app) qnext[base_q + __popc(ap & ((1u << lane) - 1u))] = myv;
            }
        }
        relaxed += (unsigned long long)cnt * __popc(m) * SPL;
    }
}

template <int SPL>
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
        int32_t du[SPL];
        load_row<SPL>(dist + (size_t)u * 32 * SPL + lane * SPL, du);
        relax_range<SPL>(nbr, w, dist, m, du, b, e, act_next, qnext, qnext_len, rel);
    }
    rel = warp_sum(rel);
    if (lane == 0 && rel) atomicAdd(relaxed, rel);
}

template <int SPL>
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
        int32_t du[SPL];
        load_row<SPL>(dist + (size_t)u * 32 * SPL + lane * SPL, du);
        relax_range<SPL>(nbr, w, dist, m, du, b, e, act_next, qnext, qnext_len, rel);
    }
    rel = warp_sum(rel);
    if (lane == 0 && rel) atomicAdd(relaxed, rel);
}

__global__ void mssp_clear(const int32_t *q, int nq, uint32_t *act) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) act[q[i]] = 0;
}

// dist[v][K] -> out[s][v] for the group's sources, 32-vertex tiles through
// shared memory (coalesced reads of rows, coalesced writes per source).
template <int SPL>
__global__ void mssp_transpose(const int32_t *dist, int32_t n, int nsrc, int32_t *out) {
    constexpr int K = 32 * SPL;
    __shared__ int32_t tile[32][K + 1];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int64_t vb = (int64_t)blockIdx.x * 32; vb < n; vb += (int64_t)gridDim.x * 32) {
        for (int r = ty; r < 32; r += 8) {
            const int64_t v = vb + r;
            for (int c = tx; c < K; c += 32) tile[r][c] = v < n ? dist[(size_t)v * K + c] : 0;
        }
        __syncthreads();
        for (int s = ty; s < nsrc; s += 8) {
            const int64_t v = vb + tx;
            if (v < n) out[(size_t)s * n + v] = tile[tx][s];
        }
        __syncthreads();
    }
}

template <int SPL>
hc_status run_group(hc_graph *g, const int32_t *h_src, int k, int32_t *dst, int max_epochs, int *epochs_out,
                    unsigned long long *relaxed) {
    constexpr int K = 32 * SPL;
    const int64_t n = g->N;
    const int64_t max_tasks = 2 * (g->M / kLongRow) + n / kLongRow + 64;
    HC_TRY(g->ws_batch.ensure((size_t)n * K * 4 + (size_t)n * 4 * 4 + sizeof(int2) * max_tasks + 8192));
    char *p = g->ws_batch.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    int32_t *dist = (int32_t *)take((size_t)n * K * 4);
    uint32_t *act[2] = {(uint32_t *)take((size_t)n * 4), (uint32_t *)take((size_t)n * 4)};
    int32_t *q[2] = {(int32_t *)take((size_t)n * 4), (int32_t *)take((size_t)n * 4)};
    int2 *tasks = (int2 *)take(sizeof(int2) * max_tasks);
    int *ctr = (int *)take(256);  // [0],[1] queue lengths, [2] tasks
    int32_t *d_src = (int32_t *)take(sizeof(int32_t) * 128);
    const int grid = g->sm_count * 8;
    HC_TRY(g->pinned.ensure(64));
    volatile int *hq = g->pinned.as<int>();
    HC_CUDA_TRY(cudaMemcpyAsync(d_src, h_src, sizeof(int32_t) * k, cudaMemcpyHostToDevice, g->stream));
    { mssp_init<SPL><<<grid, 256, 0, g->stream>>>(g->N, dist, act[0], act[1]); ::hc::count_launch(); }
    { mssp_seed<SPL><<<1, 32, 0, g->stream>>>(k, d_src, dist, act[0], q[0], &ctr[0]); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    HC_CUDA_TRY(cudaMemcpyAsync((void *)hq, &ctr[0], 4, cudaMemcpyDeviceToHost, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    int nq = *hq;
    int ep = 0;
    for (; nq > 0; ep++) {
        if (ep >= max_epochs) return fail(HC_ERR_NOT_CONVERGED, "hc_sssp_batched: epoch cap reached");
        const int c = ep & 1;
        HC_CUDA_TRY(cudaMemsetAsync(&ctr[c ^ 1], 0, 4, g->stream));
        HC_CUDA_TRY(cudaMemsetAsync(&ctr[2], 0, 4, g->stream));
        {
            mssp_epoch<SPL><<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(),
                                                         g->wgt.as<int32_t>(), dist, q[c], nq, act[c], act[c ^ 1],
                                                         q[c ^ 1], &ctr[c ^ 1], tasks, &ctr[2], relaxed);
            ::hc::count_launch();
        }
        {
            mssp_tasks<SPL><<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(),
                                                         g->wgt.as<int32_t>(), dist, tasks, &ctr[2], act[c],
                                                         act[c ^ 1], q[c ^ 1], &ctr[c ^ 1], relaxed);
            ::hc::count_launch();
        }
        { mssp_clear<<<(nq + 255) / 256, 256, 0, g->stream>>>(q[c], nq, act[c]); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        HC_CUDA_TRY(cudaMemcpyAsync((void *)hq, &ctr[c ^ 1], 4, cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        nq = *hq;
    }
    *epochs_out = ep;
    if (dst) {
        { mssp_transpose<SPL><<<grid, 256, 0, g->stream>>>(dist, g->N, k, dst); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
    }
    return HC_OK;
}

}  // namespace
}  // namespace hc

using namespace hc;

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
    // Group width: 32, 64 or 128 sources (0 = the default 128).
    const int group = o.group <= 0 ? 128 : (o.group <= 32 ? 32 : (o.group <= 64 ? 64 : 128));
    const int64_t n = g->N;
    const bool dev_out = is_device_pointer(dist_out);
    if (dist_out && !dev_out) HC_TRY(g->ws_out0.ensure(sizeof(int32_t) * (size_t)group * n));
    const int max_epochs = o.max_epochs > 0 ? o.max_epochs : 0x7fffffff;
    HC_TRY(g->ws_src.ensure(64));
    unsigned long long *relaxed = g->ws_src.as<unsigned long long>();
    HC_CUDA_TRY(cudaMemsetAsync(relaxed, 0, 8, g->stream));
    HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    int epochs_max = 0, groups = 0;
    for (int s0 = 0; s0 < num_sources; s0 += group, groups++) {
        const int k = std::min(group, num_sources - s0);
        int32_t *dst = nullptr;
        if (dist_out) dst = dev_out ? dist_out + (size_t)s0 * n : g->ws_out0.as<int32_t>();
        int ep = 0;
        if (group == 32) HC_TRY(run_group<1>(g, src.data() + s0, k, dst, max_epochs, &ep, relaxed));
        else if (group == 64) HC_TRY(run_group<2>(g, src.data() + s0, k, dst, max_epochs, &ep, relaxed));
        else HC_TRY(run_group<4>(g, src.data() + s0, k, dst, max_epochs, &ep, relaxed));
        if (dist_out && !dev_out)
            HC_TRY(copy_out(dist_out + (size_t)s0 * n, dst, sizeof(int32_t) * (size_t)k * n, g->stream));
        epochs_max = std::max(epochs_max, ep);
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
        // group's 32 lanes, plus the 4 B distance read per source relaxed.
        stats->bytes_model = (double)rel / (32.0 * (group / 32)) * 8.0 + (double)rel * 4.0;
    }
    return HC_OK;
}
