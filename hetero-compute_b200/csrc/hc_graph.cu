// Device graph handle: upload, validation, degree analysis and the derived
// arrays PageRank needs.  Replaces the per-call cudaMalloc + H2D of the
// reference drivers (src/kernels/gpu/sssp.cuh:51-61, src/graph.cuh:250-286).
#include <algorithm>
#include <cstring>

#include "hc_graph.cuh"

namespace hc {

constexpr int64_t kNbrPad = 64;

bool is_device_pointer(const void *p) {
    if (!p) return false;
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

namespace {
// The graph whose derived arrays an allocation of this thread may release,
// and what its running call needs (set by ReclaimScope).
thread_local hc_graph *t_reclaim_g = nullptr;
thread_local unsigned t_reclaim_keep = 0;

// Releases what the running call does not need; true if anything was freed.
bool reclaim(hc_graph *g, unsigned keep, const DevBuf *self) {
    bool freed = false;
    auto drop = [&](DevBuf &b) {
        if (&b != self && b.ptr) {
            b.release();
            freed = true;
        }
    };
    if (!(keep & kKeepAdj) && &g->sssp_adj != self) {
        drop(g->sssp_adj);
        g->sssp_adj_ready = 0;
    }
    if (!(keep & kKeepPrOrd) && &g->pr_ord != self) {
        drop(g->pr_ord);
        g->pr_ord_levels = -1;
    }
    if (!(keep & kKeepPrWeighted) && &g->wtn != self && &g->inv_wsum != self && &g->wf32 != self) {
        drop(g->wtn);
        drop(g->inv_wsum);
        drop(g->wf32);
    }
    if (!(keep & kKeepBatch)) drop(g->ws_batch);
    return freed;
}
}  // namespace

ReclaimScope::ReclaimScope(hc_graph *g, unsigned keep) : prev_g(t_reclaim_g), prev_keep(t_reclaim_keep) {
    t_reclaim_g = g;
    t_reclaim_keep = keep;
}

ReclaimScope::~ReclaimScope() {
    t_reclaim_g = prev_g;
    t_reclaim_keep = prev_keep;
}

hc_status DevBuf::ensure(size_t want) {
    if (want <= bytes && ptr) return HC_OK;
    release();
    size_t b = std::max<size_t>(want, 256);
    cudaError_t e = cudaMalloc(&ptr, b);
    if (e == cudaErrorMemoryAllocation && t_reclaim_g && reclaim(t_reclaim_g, t_reclaim_keep, this)) {
        cudaGetLastError();
        e = cudaMalloc(&ptr, b);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return fail(HC_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", b, cudaGetErrorString(e));
    }
    bytes = b;
    return HC_OK;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

hc_status PinnedBuf::ensure(size_t want) {
    if (want <= bytes && ptr) return HC_OK;
    release();
    size_t b = std::max<size_t>(want, 4096);
    cudaError_t e = cudaMallocHost(&ptr, b);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return fail(HC_ERR_OOM, "cudaMallocHost of %zu bytes failed: %s", b, cudaGetErrorString(e));
    }
    bytes = b;
    return HC_OK;
}

void PinnedBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

hc_status copy_in(void *dst_dev, const void *src_any, size_t bytes, cudaStream_t s) {
    if (!bytes) return HC_OK;
    HC_CUDA_TRY(cudaMemcpyAsync(dst_dev, src_any, bytes, cudaMemcpyDefault, s));
    return HC_OK;
}

hc_status copy_out(void *dst_any, const void *src_dev, size_t bytes, cudaStream_t s) {
    if (!bytes) return HC_OK;
    HC_CUDA_TRY(cudaMemcpyAsync(dst_any, src_dev, bytes, cudaMemcpyDefault, s));
    return HC_OK;
}

hc_status OutPipe::init(hc_graph *graph, int arrays, size_t each) {
    g = graph;
    narr = arrays;
    bytes = each;
    copy_bytes = each;
    pending = false;
    if (!g->copy_stream) HC_CUDA_TRY(cudaStreamCreateWithFlags(&g->copy_stream, cudaStreamNonBlocking));
    for (int s = 0; s < 2; s++) {
        if (!g->ev_ready[s]) HC_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_ready[s], cudaEventDisableTiming));
        if (!g->ev_done[s]) {
            HC_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_done[s], cudaEventDisableTiming));
            HC_CUDA_TRY(cudaEventRecord(g->ev_done[s], g->copy_stream));  // nothing to wait for yet
        }
        for (int j = 0; j < arrays; j++) HC_TRY(g->ws_stage[s][j].ensure(each));
    }
    return HC_OK;
}

hc_status OutPipe::acquire(int i, int32_t **bufs) {
    HC_TRY(flush());
    const int s = i & 1;
    HC_CUDA_TRY(cudaStreamWaitEvent(g->stream, g->ev_done[s], 0));
    for (int j = 0; j < narr; j++) bufs[j] = g->ws_stage[s][j].as<int32_t>();
    return HC_OK;
}

hc_status OutPipe::release(int i, void *const *dst) {
    const int s = i & 1;
    HC_CUDA_TRY(cudaEventRecord(g->ev_ready[s], g->stream));
    pending = true;
    pend_slot = s;
    for (int j = 0; j < narr; j++) pend_dst[j] = dst[j];
    return HC_OK;
}

hc_status OutPipe::flush() {
    if (!pending) return HC_OK;
    pending = false;
    const int s = pend_slot;
    HC_CUDA_TRY(cudaStreamWaitEvent(g->copy_stream, g->ev_ready[s], 0));
    for (int j = 0; j < narr; j++)
        if (pend_dst[j])
            HC_CUDA_TRY(cudaMemcpyAsync(pend_dst[j], g->ws_stage[s][j].ptr, copy_bytes, cudaMemcpyDefault,
                                        g->copy_stream));
    HC_CUDA_TRY(cudaEventRecord(g->ev_done[s], g->copy_stream));
    return HC_OK;
}

hc_status OutPipe::finish() {
    HC_TRY(flush());
    HC_CUDA_TRY(cudaStreamSynchronize(g->copy_stream));
    return HC_OK;
}

namespace {
__global__ void words_zero(uint32_t *p, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 0u;
}
__global__ void words_to_host(uint32_t *dst, const uint32_t *src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    __threadfence_system();
}
}  // namespace

hc_status ctl_zero(hc_graph *g, void *dev, size_t bytes) {
    { words_zero<<<1, 256, 0, g->stream>>>(reinterpret_cast<uint32_t *>(dev), (int)((bytes + 3) / 4)); count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    return HC_OK;
}

hc_status ctl_read(hc_graph *g, const void *dev, size_t bytes, int slot, const void **host) {
    if (bytes > kCtlSlotBytes || slot < 0 || slot >= kCtlSlots) return fail(HC_ERR_INVALID_ARG, "ctl_read: bad slot");
    if (!g->ctl_host) {
        HC_CUDA_TRY(cudaHostAlloc(&g->ctl_host, kCtlSlotBytes * kCtlSlots, cudaHostAllocMapped));
        HC_CUDA_TRY(cudaHostGetDevicePointer(&g->ctl_host_dev, g->ctl_host, 0));
    }
    uint32_t *d = reinterpret_cast<uint32_t *>(static_cast<char *>(g->ctl_host_dev) + (size_t)slot * kCtlSlotBytes);
    { words_to_host<<<1, 256, 0, g->stream>>>(d, reinterpret_cast<const uint32_t *>(dev), (int)((bytes + 3) / 4)); count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    *host = static_cast<const char *>(g->ctl_host) + (size_t)slot * kCtlSlotBytes;
    return HC_OK;
}

hc_status activate(hc_graph *g) {
    if (!g) return fail(HC_ERR_INVALID_ARG, "null graph handle");
    HC_CUDA_TRY(cudaSetDevice(g->device));
    return HC_OK;
}

namespace {

struct Analysis {
    int unsorted;      // degrees increase somewhere
    int first_zero;    // first vertex of degree 0 (N if none)
    int max_degree;
    int first_small;   // first vertex of degree < 32 (N if none)
    int bad_index;     // offsets decrease or exceed [0, M]
    int bad_nbr;       // neighbour outside [0, N)
    int rows_unsorted; // some row not strictly increasing
    int pad;
};

__global__ void analyze_index(const int64_t *index, int32_t n, int64_t m, Analysis *out) {
    const int stride = gridDim.x * blockDim.x;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        int64_t b = index[v], e = index[v + 1];
        if (b < 0 || e < b || e > m) {
            out->bad_index = 1;
            continue;
        }
        int64_t d = e - b;
        if (v + 1 < n) {
            int64_t d2 = index[v + 2] - e;
            if (d2 > d) out->unsorted = 1;
        }
        if (d == 0) atomicMin(&out->first_zero, v);
        if (d < 32) atomicMin(&out->first_small, v);
        atomicMax(&out->max_degree, (int)(d > 0x7fffffffll ? 0x7fffffffll : d));
    }
}

// Neighbour range and row order; only run once the index checked out.
__global__ void analyze_rows(const int64_t *index, const int32_t *nbr, int32_t n, Analysis *out) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        int64_t b = index[v], e = index[v + 1];
        for (int64_t i = b + lane; i < e; i += 32) {
            int32_t x = nbr[i];
            if (x < 0 || x >= n) out->bad_nbr = 1;
            if (i + 1 < e && nbr[i + 1] <= x) out->rows_unsorted = 1;
        }
    }
}

}  // namespace

// One pass over a caller's CSR: every row [index[v], index[v+1]) inside
// [0, m], index[0] == 0, index[n] == m, and every neighbour id in [0, n).
// A row whose bounds fail is not read, so the check itself stays inside the
// arrays (index[n + 1] entries, neighbours m entries of `stride` int32 words:
// 1 for an id array, 2 for the reference's interleaved {id, weight} layout).
// Sets bit 0 of *flag for a bad offset and bit 1 for a bad neighbour id.
__global__ void csr_check(const int64_t *index, const int32_t *nbr, int stride, int32_t n, int64_t m, int *flag) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const int64_t b = index[v], e = index[v + 1];
        const bool row_ok = b >= 0 && b <= e && e <= m && (v != 0 || b == 0) && (v != n - 1 || e == m);
        if (!row_ok) {
            if (lane == 0) atomicOr(flag, 1);
            continue;
        }
        bool bad = false;
        for (int64_t i = b + lane; i < e; i += 32) {
            const int32_t x = nbr[i * stride];
            bad |= x < 0 || x >= n;
        }
        if (__any_sync(kFull, bad) && lane == 0) atomicOr(flag, 2);
    }
}

hc_status csr_check_async(const int64_t *index, const int32_t *nbr, int stride, int32_t n, int64_t m, int *flag_dev,
                          int sm_count, cudaStream_t s) {
    HC_CUDA_TRY(cudaMemsetAsync(flag_dev, 0, sizeof(int), s));
    if (n < 1) return HC_OK;
    const int blocks = (int)std::min<int64_t>((int64_t)sm_count * 8, ((int64_t)n + 7) / 8);
    { csr_check<<<blocks, 256, 0, s>>>(index, nbr, stride, n, m, flag_dev); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    return HC_OK;
}

namespace {

__global__ void build_inv_deg(const int64_t *index, int32_t n, float *inv_deg) {
    const int stride = gridDim.x * blockDim.x;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        int64_t d = index[v + 1] - index[v];
        inv_deg[v] = d ? 1.0f / (float)d : 0.0f;
    }
}

// Row sums of the raw weights (warp per row), stored as reciprocals.
__global__ void build_inv_wsum(const int64_t *index, const float *w, int32_t n, float *inv_wsum) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        int64_t b = index[v], e = index[v + 1];
        double s = 0.0;
        for (int64_t i = b + lane; i < e; i += 32) s += (double)w[i];
        s = warp_sum(s);
        if (lane == 0) inv_wsum[v] = s > 0.0 ? (float)(1.0 / s) : 0.0f;
    }
}

__global__ void weights_to_f32(const int32_t *w, size_t n, float *out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)w[i];
}

// wtn[slot (v,i)] = w[u -> v] / sum_k w[u -> k] with u = nbr[v][i]: the weight
// the forward pull at v needs, stored in v's own row so the pull streams it.
// Rows are sorted, so the reverse slot is found by binary search in row u.
__global__ void build_wtn(const int64_t *index, const int32_t *nbr, const float *w,
                          const float *inv_wsum, int32_t n, float *wtn, int *missing) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        int64_t b = index[v], e = index[v + 1];
        for (int64_t i = b + lane; i < e; i += 32) {
            int32_t u = nbr[i];
            int64_t lo = index[u], hi = index[u + 1];
            while (lo < hi) {
                int64_t mid = (lo + hi) >> 1;
                if (nbr[mid] < v) lo = mid + 1; else hi = mid;
            }
            if (lo < index[u + 1] && nbr[lo] == v) {
                wtn[i] = w[lo] * inv_wsum[u];
            } else {
                wtn[i] = 0.0f;
                *missing = 1;
            }
        }
    }
}

}  // namespace

// Edge-multiset hashing: each edge v->u (v != u) hashes its unordered key
// (min, max) -- and, for the weighted sums, its weight bits -- and adds the
// hash to the "lo" sum when v < u, else to the "hi" sum.  The edge multiset
// equals its reverse exactly when every lo sum equals its hi sum, up to a
// collision of two independent 64-bit hashes (SplitMix64 finaliser, Steele et
// al. 2014) of wrapping sums.  One streaming pass, no searches, any row order.
__device__ __forceinline__ uint64_t mix_u64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void edge_hash_sums(const int64_t *index, const int32_t *nbr, const uint32_t *wbits, int32_t n,
                               unsigned long long *acc) {
    __shared__ unsigned long long s_red[32];
    unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // {struct, weight} x {hash a, hash b} x {lo, hi}
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const int64_t b = index[v], e = index[v + 1];
        for (int64_t i = b + lane; i < e; i += 32) {
            const int32_t u = nbr[i];
            if (u == v) continue;
            const uint64_t lo = (uint64_t)(uint32_t)min(u, v), hi = (uint64_t)(uint32_t)max(u, v);
            const uint64_t key = (lo << 32) | hi;
            const int side = v < u ? 0 : 1;
            const uint64_t ha = mix_u64(key + 0x9e3779b97f4a7c15ull);
            const uint64_t hb = mix_u64(key ^ 0xd1b54a32d192ed03ull);
            h[0 + side] += ha;
            h[2 + side] += hb;
            if (wbits) {
                const uint64_t wk = mix_u64((uint64_t)wbits[i] + 0x632be59bd9b4e019ull);
                h[4 + side] += mix_u64(ha ^ wk);
                h[6 + side] += mix_u64(hb + wk);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const unsigned long long t = block_sum(h[j], s_red);
        if (threadIdx.x == 0 && t) atomicAdd(acc + j, t);
    }
}

hc_status edge_symmetry(hc_graph *g, const uint32_t *wbits, bool *structure, bool *weights) {
    DevBuf acc;
    HC_TRY(acc.ensure(8 * sizeof(unsigned long long)));
    HC_CUDA_TRY(cudaMemsetAsync(acc.ptr, 0, 8 * sizeof(unsigned long long), g->stream));
    { edge_hash_sums<<<g->sm_count * 8, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(), wbits, g->N,
                                                             acc.as<unsigned long long>()); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    unsigned long long h[8];
    HC_CUDA_TRY(cudaMemcpyAsync(h, acc.ptr, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    *structure = h[0] == h[1] && h[2] == h[3];
    *weights = *structure && (!wbits || (h[4] == h[5] && h[6] == h[7]));
    return HC_OK;
}

hc_status ensure_pr_symmetry(hc_graph *g, bool weighted, bool *symmetric) {
    if (g->pr_sym_struct < 0 || (weighted && g->pr_sym_w < 0)) {
        const uint32_t *w = weighted ? reinterpret_cast<const uint32_t *>(pr_weights(g)) : nullptr;
        bool st = false, ws = false;
        HC_TRY(edge_symmetry(g, w, &st, &ws));
        g->pr_sym_struct = st;
        if (weighted) g->pr_sym_w = ws;
    }
    *symmetric = weighted ? g->pr_sym_w == 1 : g->pr_sym_struct == 1;
    return HC_OK;
}

const float *pr_weights(const hc_graph *g) {
    return g->wtype == HC_W_I32 ? g->wf32.as<float>() : g->wgt.as<float>();
}

hc_status ensure_pr_derived(hc_graph *g, bool weighted) {
    const int grid = g->sm_count * 8, block = 256;
    if (!g->inv_deg.ptr) {
        HC_TRY(g->inv_deg.ensure(sizeof(float) * std::max<int32_t>(g->N, 1)));
        { build_inv_deg<<<grid, block, 0, g->stream>>>(g->index.as<int64_t>(), g->N, g->inv_deg.as<float>()); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
    }
    if (weighted && !g->wtn.ptr) {
        if (g->wtype == HC_W_NONE) return fail(HC_ERR_UNSUPPORTED, "weighted PageRank needs edge weights");
        if (g->wtype == HC_W_I32 && !g->wf32.ptr) {
            // Exact for |w| < 2^24 (the generators' int32 weights are in [1, 255]).
            HC_TRY(g->wf32.ensure(sizeof(float) * (size_t)(g->M + kNbrPad)));
            { weights_to_f32<<<grid, block, 0, g->stream>>>(g->wgt.as<int32_t>(), (size_t)(g->M + kNbrPad),
                                                            g->wf32.as<float>()); ::hc::count_launch(); }
            HC_CUDA_TRY(cudaGetLastError());
        }
        HC_TRY(g->inv_wsum.ensure(sizeof(float) * std::max<int32_t>(g->N, 1)));
        HC_TRY(g->wtn.ensure(sizeof(float) * (size_t)(g->M + kNbrPad)));
        { build_inv_wsum<<<grid, block, 0, g->stream>>>(g->index.as<int64_t>(), pr_weights(g), g->N,
                                                        g->inv_wsum.as<float>()); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        DevBuf flag;
        HC_TRY(flag.ensure(sizeof(int)));
        HC_CUDA_TRY(cudaMemsetAsync(flag.ptr, 0, sizeof(int), g->stream));
        { build_wtn<<<grid, block, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(),
                                                   pr_weights(g), g->inv_wsum.as<float>(), g->N,
                                                   g->wtn.as<float>(), flag.as<int>()); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        int missing = 0;
        HC_CUDA_TRY(cudaMemcpyAsync(&missing, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        flag.release();
        if (missing) {
            g->wtn.release();
            return fail(HC_ERR_INVALID_ARG,
                        "weighted PageRank needs a symmetric structure with sorted rows "
                        "(an edge u->v has no v->u slot)");
        }
    }
    return HC_OK;
}

}  // namespace hc

int64_t hc_graph::bytes_held() const {
    const hc::DevBuf *bufs[] = {&index, &nbr, &wgt, &inv_deg, &inv_wsum, &wtn, &wf32, &pr_plan,
                                &pr_plan_huge_rows, &pr_ord, &ws_bfs, &ws_sssp, &ws_pr, &ws_batch,
                                &ws_out0, &ws_out1, &ws_ctl, &ws_plan_ms, &ws_plan_mssp, &ws_src, &sssp_adj};
    int64_t t = 0;
    for (auto *b : bufs) t += (int64_t)b->bytes;
    for (int s = 0; s < 2; s++)
        for (int j = 0; j < 2; j++) t += (int64_t)ws_stage[s][j].bytes;
    return t;
}

namespace hc {

hc_status graph_alloc(int32_t num_nodes, int64_t num_edges, hc_wtype wtype, int32_t device, hc_graph **out) {
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(HC_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (device < 0 || device >= ndev) return fail(HC_ERR_INVALID_ARG, "device %d out of range (%d)", device, ndev);
    HC_CUDA_TRY(cudaSetDevice(device));
    hc_graph *g = new hc_graph();
    g->device = device;
    g->N = num_nodes;
    g->M = num_edges;
    g->wtype = wtype;
    auto bail = [&](hc_status s) {
        hc_graph_destroy(g);
        return s;
    };
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return bail(fail(HC_ERR_CUDA, "cudaGetDeviceProperties failed"));
    g->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(HC_ERR_CUDA, "cudaStreamCreate failed"));
    g->stream = g->own_stream;
    if (cudaEventCreate(&g->ev_start) != cudaSuccess || cudaEventCreate(&g->ev_stop) != cudaSuccess)
        return bail(fail(HC_ERR_CUDA, "cudaEventCreate failed"));
    hc_status st;
    if ((st = g->index.ensure(sizeof(int64_t) * ((size_t)num_nodes + 1))) != HC_OK) return bail(st);
    if ((st = g->nbr.ensure(sizeof(int32_t) * (size_t)(num_edges + kNbrPad))) != HC_OK) return bail(st);
    if (cudaMemsetAsync(g->nbr.ptr, 0, g->nbr.bytes, g->stream) != cudaSuccess)
        return bail(fail(HC_ERR_CUDA, "memset failed"));
    if (wtype != HC_W_NONE) {
        if ((st = g->wgt.ensure(4 * (size_t)(num_edges + kNbrPad))) != HC_OK) return bail(st);
        if (cudaMemsetAsync(g->wgt.ptr, 0, g->wgt.bytes, g->stream) != cudaSuccess)
            return bail(fail(HC_ERR_CUDA, "memset failed"));
    }
    *out = g;
    return HC_OK;
}

hc_status graph_finish(hc_graph *g, const char *who) {
    const int32_t num_nodes = g->N;
    const int64_t num_edges = g->M;
    // Validate and analyse on the device.
    DevBuf abuf;
    HC_TRY(abuf.ensure(sizeof(Analysis)));
    Analysis init;
    std::memset(&init, 0, sizeof(init));
    init.first_zero = num_nodes;
    init.first_small = num_nodes;
    int64_t ends[2] = {0, 0};
    if (cudaMemcpyAsync(abuf.ptr, &init, sizeof(init), cudaMemcpyHostToDevice, g->stream) != cudaSuccess ||
        cudaMemcpyAsync(&ends[0], g->index.as<int64_t>(), 8, cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
        cudaMemcpyAsync(&ends[1], g->index.as<int64_t>() + num_nodes, 8, cudaMemcpyDeviceToHost, g->stream) != cudaSuccess)
        return fail(HC_ERR_CUDA, "%s: analysis setup failed", who);
    const int grid = g->sm_count * 8;
    { analyze_index<<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), num_nodes, num_edges, abuf.as<Analysis>()); ::hc::count_launch(); }
    Analysis res;
    if (cudaMemcpyAsync(&res, abuf.ptr, sizeof(res), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
        cudaStreamSynchronize(g->stream) != cudaSuccess)
        return fail(HC_ERR_CUDA, "%s: graph analysis failed: %s", who, cudaGetErrorString(cudaGetLastError()));
    if (ends[0] != 0 || ends[1] != num_edges || res.bad_index)
        return fail(HC_ERR_INVALID_ARG, "%s: index must be non-decreasing from 0 to num_edges", who);
    { analyze_rows<<<grid, 256, 0, g->stream>>>(g->index.as<int64_t>(), g->nbr.as<int32_t>(), num_nodes,
                                                abuf.as<Analysis>()); ::hc::count_launch(); }
    if (cudaMemcpyAsync(&res, abuf.ptr, sizeof(res), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
        cudaStreamSynchronize(g->stream) != cudaSuccess)
        return fail(HC_ERR_CUDA, "%s: graph analysis failed: %s", who, cudaGetErrorString(cudaGetLastError()));
    if (res.bad_nbr) return fail(HC_ERR_INVALID_ARG, "%s: neighbour id outside [0, N)", who);
    g->degree_sorted = !res.unsorted;
    g->rows_sorted = !res.rows_unsorted;
    g->max_degree = res.max_degree;
    g->n_active = g->degree_sorted ? res.first_zero : num_nodes;
    if (g->degree_sorted) {
        int32_t r = (int32_t)std::min<int64_t>(((int64_t)res.first_small + 31) / 32 * 32, num_nodes);
        g->n_warp_rows = r;
    } else {
        g->n_warp_rows = 0;
    }
    return HC_OK;
}

}  // namespace hc

using namespace hc;

extern "C" {

hc_status hc_graph_create(const int64_t *index, const int32_t *neighbors, const void *weights,
                          hc_wtype wtype, int32_t num_nodes, int64_t num_edges, int32_t device,
                          hc_graph **out) {
    clear_error();
    if (!out) return fail(HC_ERR_INVALID_ARG, "hc_graph_create: null output handle");
    *out = nullptr;
    if (!index || num_nodes < 1 || num_edges < 0 || (num_edges > 0 && !neighbors))
        return fail(HC_ERR_INVALID_ARG, "hc_graph_create: bad CSR (N=%d, M=%lld)", num_nodes,
                    (long long)num_edges);
    if (wtype != HC_W_NONE && !weights)
        return fail(HC_ERR_INVALID_ARG, "hc_graph_create: weight type given without weights");
    hc_graph *g = nullptr;
    HC_TRY(graph_alloc(num_nodes, num_edges, wtype, device, &g));
    auto bail = [&](hc_status s) {
        hc_graph_destroy(g);
        return s;
    };
    hc_status st;
    if ((st = copy_in(g->index.ptr, index, sizeof(int64_t) * ((size_t)num_nodes + 1), g->stream)) != HC_OK)
        return bail(st);
    if ((st = copy_in(g->nbr.ptr, neighbors, sizeof(int32_t) * (size_t)num_edges, g->stream)) != HC_OK)
        return bail(st);
    if (wtype != HC_W_NONE && (st = copy_in(g->wgt.ptr, weights, 4 * (size_t)num_edges, g->stream)) != HC_OK)
        return bail(st);
    if ((st = graph_finish(g, "hc_graph_create")) != HC_OK) return bail(st);
    *out = g;
    return HC_OK;
}

hc_status hc_csr_check(const int64_t *index, const void *neighbors, int32_t interleaved, int32_t num_nodes,
                       int64_t num_edges, void *stream) {
    clear_error();
    if (!index || num_nodes < 1 || num_edges < 0 || (num_edges > 0 && !neighbors))
        return fail(HC_ERR_INVALID_ARG, "hc_csr_check: bad arguments (N=%d, M=%lld)", num_nodes, (long long)num_edges);
    if (!is_device_pointer(index) || (num_edges > 0 && !is_device_pointer(neighbors)))
        return fail(HC_ERR_INVALID_ARG, "hc_csr_check: index and neighbours must be device memory");
    int dev = 0, sms = 0;
    HC_CUDA_TRY(cudaGetDevice(&dev));
    HC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevBuf flag;
    HC_TRY(flag.ensure(sizeof(int)));
    HC_TRY(csr_check_async(index, static_cast<const int32_t *>(neighbors), interleaved ? 2 : 1, num_nodes, num_edges,
                           flag.as<int>(), sms, s));
    int h = 0;
    HC_CUDA_TRY(cudaMemcpyAsync(&h, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    HC_CUDA_TRY(cudaStreamSynchronize(s));
    if (h & 1) return fail(HC_ERR_INVALID_ARG, "hc_csr_check: offsets must rise from 0 to num_edges");
    if (h & 2) return fail(HC_ERR_INVALID_ARG, "hc_csr_check: neighbour id outside [0, num_nodes)");
    return HC_OK;
}

hc_status hc_graph_destroy(hc_graph *g) {
    if (!g) return HC_OK;
    cudaSetDevice(g->device);
    if (g->own_stream) cudaStreamSynchronize(g->own_stream);
    if (g->stream && g->stream != g->own_stream) cudaStreamSynchronize(g->stream);
    DevBuf *bufs[] = {&g->index, &g->nbr, &g->wgt, &g->inv_deg, &g->inv_wsum, &g->wtn, &g->wf32, &g->pr_plan,
                      &g->pr_plan_huge_rows, &g->ws_bfs, &g->ws_sssp, &g->ws_pr, &g->ws_batch,
                      &g->ws_out0, &g->ws_out1, &g->ws_ctl, &g->ws_plan_ms, &g->ws_plan_mssp, &g->ws_src,
                      &g->sssp_adj, &g->pr_ord};
    for (auto *b : bufs) b->release();
    if (g->copy_stream) cudaStreamSynchronize(g->copy_stream);
    for (int s = 0; s < 2; s++) {
        for (int j = 0; j < 2; j++) g->ws_stage[s][j].release();
        if (g->ev_ready[s]) cudaEventDestroy(g->ev_ready[s]);
        if (g->ev_done[s]) cudaEventDestroy(g->ev_done[s]);
    }
    if (g->copy_stream) cudaStreamDestroy(g->copy_stream);
    g->pinned.release();
    if (g->ctl_host) cudaFreeHost(g->ctl_host);
    if (g->ev_start) cudaEventDestroy(g->ev_start);
    if (g->ev_stop) cudaEventDestroy(g->ev_stop);
    if (g->own_stream) cudaStreamDestroy(g->own_stream);
    delete g;
    return HC_OK;
}

hc_status hc_graph_set_stream(hc_graph *g, void *stream) {
    clear_error();
    if (!g) return fail(HC_ERR_INVALID_ARG, "null graph handle");
    g->stream = stream ? (cudaStream_t)stream : g->own_stream;
    return HC_OK;
}

hc_status hc_graph_get_info(const hc_graph *g, hc_graph_info *info) {
    clear_error();
    if (!g || !info) return fail(HC_ERR_INVALID_ARG, "null argument");
    info->num_nodes = g->N;
    info->num_edges = g->M;
    info->num_active = g->n_active;
    info->degree_sorted = g->degree_sorted;
    info->max_degree = g->max_degree;
    info->device = g->device;
    info->wtype = g->wtype;
    info->device_bytes = g->bytes_held();
    return HC_OK;
}

}  // extern "C"

extern "C" {

hc_status hc_dev_malloc(void **ptr, size_t bytes, int32_t device) {
    clear_error();
    if (!ptr) return fail(HC_ERR_INVALID_ARG, "hc_dev_malloc: null output");
    *ptr = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(HC_ERR_NO_DEVICE, "hc_dev_malloc: no CUDA device visible");
    }
    if (device < 0 || device >= ndev) return fail(HC_ERR_INVALID_ARG, "hc_dev_malloc: bad device %d", device);
    HC_CUDA_TRY(cudaSetDevice(device));
    HC_CUDA_TRY(cudaMalloc(ptr, bytes ? bytes : 1));
    return HC_OK;
}

hc_status hc_dev_free(void *ptr) {
    clear_error();
    if (ptr) HC_CUDA_TRY(cudaFree(ptr));
    return HC_OK;
}

hc_status hc_memcpy(void *dst, const void *src, size_t bytes) {
    clear_error();
    if (!bytes) return HC_OK;
    if (!dst || !src) return fail(HC_ERR_INVALID_ARG, "hc_memcpy: null pointer");
    HC_CUDA_TRY(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
    return HC_OK;
}

hc_status hc_dev_memset(void *ptr, int32_t value, size_t bytes) {
    clear_error();
    if (!bytes) return HC_OK;
    if (!ptr) return fail(HC_ERR_INVALID_ARG, "hc_dev_memset: null pointer");
    HC_CUDA_TRY(cudaMemset(ptr, value, bytes));
    return HC_OK;
}

hc_status hc_device_synchronize(void) {
    clear_error();
    HC_CUDA_TRY(cudaDeviceSynchronize());
    return HC_OK;
}

}  // extern "C"
