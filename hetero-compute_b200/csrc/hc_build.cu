// Synthetic graphs built on the device: the same CSR as hc_gen_kronecker /
// hc_gen_uniform (hc_host.cpp) followed by hc_graph_create, with the edge
// streams of hc_gen.h, so no host build, host memory or upload is needed.
//
// Steps, each the device form of the host builder's pass:
//   1. count the symmetrised degree of every vertex (self-loops dropped);
//   2. offsets by an exclusive scan;
//   3. scatter both directions of every pair as (neighbour << 32 | weight);
//   4. sort every row (segmented sort, in batches below 2^30 entries);
//   5. keep the first of each neighbour run (the lightest duplicate);
//   6. new id = rank by (degree desc, old id desc): one radix sort of
//      ((max degree - degree) << 32 | (N - 1 - id));
//   7. rows in the new order with renamed neighbours, sorted again;
//   8. split into neighbour and weight arrays and hand them to
//      hc_graph_create (validation, analysis, its own copy).
// Sorting uses CUB (shipped with the CUDA toolkit); the rest are kernels here.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <vector>

#include "hc_gen.h"
#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr int64_t kSortBatch = (int64_t)1 << 30;  // entries per segmented-sort call (int counts)

template <class Pairs>
__global__ void b_count(Pairs pairs, int64_t np, unsigned long long *cnt) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < np; e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t s, d;
        pairs(e, s, d);
        if (s == d) continue;
        atomicAdd(cnt + s, 1ull);
        atomicAdd(cnt + d, 1ull);
    }
}

template <class Pairs>
__global__ void b_scatter(Pairs pairs, int64_t np, const unsigned long long *off, unsigned long long *pos,
                          hc_wtype wt, uint64_t seed, uint64_t *packed) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < np; e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t s, d;
        pairs(e, s, d);
        if (s == d) continue;
        const uint64_t w = weight_bits(wt, seed, e);
        const unsigned long long ps = off[s] + atomicAdd(pos + s, 1ull);
        const unsigned long long pd = off[d] + atomicAdd(pos + d, 1ull);
        packed[ps] = ((uint64_t)d << 32) | w;
        packed[pd] = ((uint64_t)s << 32) | w;
    }
}

// rel[i] = off[r0 + i] - off[r0], the batch's row offsets relative to its first entry.
__global__ void b_rel_offsets(const unsigned long long *off, int64_t r0, int64_t nrows, int *rel) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= nrows; i += (int64_t)gridDim.x * blockDim.x)
        rel[i] = (int)(off[r0 + i] - off[r0]);
}

// Per row (a warp): keep the first entry of each neighbour run, in place;
// ndeg = entries kept.  An entry is written at a position no later than the
// one it was read from, so a row compacts in order without losing data.
__global__ void b_dedup(const unsigned long long *off, int32_t n, uint64_t *rows, unsigned long long *ndeg,
                        unsigned long long *maxdeg) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long my_max = 0;
    for (int32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const int64_t b = (int64_t)off[v], e = (int64_t)off[v + 1];
        int64_t kept = 0;
        uint32_t carry = 0xffffffffu;  // neighbour of the previous entry (none yet)
        for (int64_t base = b; base < e; base += 32) {
            const int64_t i = base + lane;
            uint64_t x = 0;
            if (i < e) x = rows[i];
            const uint32_t nb = (uint32_t)(x >> 32);
            uint32_t prev = __shfl_up_sync(kFull, nb, 1);
            if (lane == 0) prev = carry;
            const bool keep = i < e && (i == b || nb != prev);
            const unsigned bal = __ballot_sync(kFull, keep);
            if (keep) rows[b + kept + __popc(bal & ((1u << lane) - 1u))] = x;
            kept += __popc(bal);
            const int last = (int)((e - base) < 32 ? (e - base) : 32) - 1;
            carry = __shfl_sync(kFull, nb, last);
        }
        if (lane == 0) {
            ndeg[v] = (unsigned long long)kept;
            my_max = my_max > (unsigned long long)kept ? my_max : (unsigned long long)kept;
        }
    }
    if (lane == 0 && my_max) atomicMax(maxdeg, my_max);
}

__global__ void b_rank_keys(const unsigned long long *ndeg, int32_t n, const unsigned long long *maxdeg,
                            uint64_t *keys, int32_t *ids) {
    const unsigned long long mx = *maxdeg;
    for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        keys[v] = ((uint64_t)(mx - ndeg[v]) << 32) | (uint32_t)(n - 1 - v);
        ids[v] = v;
    }
}

__global__ void b_rank(const int32_t *order, int32_t n, const unsigned long long *ndeg, int32_t *rank,
                       unsigned long long *deg_new) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t v = order[i];
        rank[v] = i;
        deg_new[i] = ndeg[v];
    }
}

// Row v (deduplicated, at off[v]) goes to row rank[v] (at noff) with every
// neighbour renamed; weights ride along in the low word.
__global__ void b_rename(const unsigned long long *off, const unsigned long long *ndeg, const int32_t *rank,
                         const uint64_t *rows, const unsigned long long *noff, int32_t n, uint64_t *out) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const uint64_t *src = rows + off[v];
        uint64_t *dst = out + noff[rank[v]];
        const int64_t d = (int64_t)ndeg[v];
        for (int64_t j = lane; j < d; j += 32) {
            const uint64_t x = src[j];
            dst[j] = ((uint64_t)(uint32_t)rank[x >> 32] << 32) | (x & 0xffffffffull);
        }
    }
}

__global__ void b_split(const uint64_t *rows, int64_t m, int32_t *nbr, uint32_t *w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t x = rows[i];
        nbr[i] = (int32_t)(x >> 32);
        if (w) w[i] = (uint32_t)x;
    }
}

__global__ void b_to_i64(const unsigned long long *in, int64_t n, int64_t *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int64_t)in[i];
}

template <class T>
T read1(const T *p) {
    T v{};
    cudaMemcpy(&v, p, sizeof(T), cudaMemcpyDeviceToHost);
    return v;
}

struct Builder {
    int grid = 0;
    cudaStream_t st = nullptr;
    DevBuf temp;  // CUB scratch, grown on demand

    hc_status scan(const unsigned long long *in, unsigned long long *out, int64_t count) {
        size_t bytes = 0;
        HC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)count, st));
        HC_TRY(temp.ensure(bytes));
        HC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(temp.ptr, bytes, in, out, (int)count, st));
        return HC_OK;
    }

    // Sorts every row [off[v], off[v+1]) of `in` into `out`, rows batched so a
    // call holds at most kSortBatch entries (a longer row is a batch of its own).
    hc_status sort_rows(const unsigned long long *off, int32_t n, const uint64_t *in, uint64_t *out, DevBuf &rel) {
        std::vector<unsigned long long> hoff((size_t)n + 1);
        HC_CUDA_TRY(cudaMemcpy(hoff.data(), off, sizeof(unsigned long long) * ((size_t)n + 1),
                               cudaMemcpyDeviceToHost));
        HC_TRY(rel.ensure(sizeof(int) * ((size_t)n + 2)));
        int64_t r0 = 0;
        while (r0 < n) {
            // Largest r1 with off[r1] - off[r0] <= kSortBatch (at least one row).
            const auto it = std::upper_bound(hoff.begin() + r0 + 1, hoff.end(), hoff[r0] + (uint64_t)kSortBatch);
            int64_t r1 = (int64_t)(it - hoff.begin()) - 1;
            if (r1 <= r0) r1 = r0 + 1;
            const int64_t items = (int64_t)(hoff[r1] - hoff[r0]);
            if (items > 0x7fffffff) return fail(HC_ERR_UNSUPPORTED, "graph build: a row of %lld entries", (long long)items);
            if (items > 0) {
                const int64_t rows = r1 - r0;
                { b_rel_offsets<<<grid, 256, 0, st>>>(off, r0, rows, rel.as<int>()); ::hc::count_launch(); }
                size_t bytes = 0;
                const int *rb = rel.as<int>();
                HC_CUDA_TRY(cub::DeviceSegmentedSort::SortKeys(nullptr, bytes, in + hoff[r0], out + hoff[r0], (int)items,
                                                              (int)rows, rb, rb + 1, st));
                HC_TRY(temp.ensure(bytes));
                HC_CUDA_TRY(cub::DeviceSegmentedSort::SortKeys(temp.ptr, bytes, in + hoff[r0], out + hoff[r0],
                                                              (int)items, (int)rows, rb, rb + 1, st));
                ::hc::count_launch();
            }
            r0 = r1;
        }
        return HC_OK;
    }
};

template <class Pairs>
hc_status build_device(const Pairs &pairs, int scale, int64_t np, hc_wtype wt, uint64_t seed, int32_t device,
                       hc_graph **out) {
    const int64_t n = (int64_t)1 << scale;
    if (n > 0x7fffffffll) return fail(HC_ERR_INVALID_ARG, "graph build: scale %d too large for int32 ids", scale);
    HC_CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    HC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    Builder B;
    B.grid = sms * 8;
    HC_CUDA_TRY(cudaStreamCreateWithFlags(&B.st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{B.st};
    const int grid = B.grid;
    cudaStream_t st = B.st;

    // 1-2. degrees and offsets.
    DevBuf cnt, off, pos;
    HC_TRY(cnt.ensure(sizeof(unsigned long long) * ((size_t)n + 1)));
    HC_TRY(off.ensure(sizeof(unsigned long long) * ((size_t)n + 1)));
    HC_CUDA_TRY(cudaMemsetAsync(cnt.ptr, 0, cnt.bytes, st));
    { b_count<<<grid, 256, 0, st>>>(pairs, np, cnt.as<unsigned long long>()); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    HC_TRY(B.scan(cnt.as<unsigned long long>(), off.as<unsigned long long>(), n + 1));
    HC_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m_raw = (int64_t)read1(off.as<unsigned long long>() + n);

    // 3. both directions of every pair.
    DevBuf packed, sorted, rel;
    HC_TRY(packed.ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(m_raw, 1)));
    HC_TRY(sorted.ensure(sizeof(uint64_t) * (size_t)std::max<int64_t>(m_raw, 1)));
    HC_CUDA_TRY(cudaMemsetAsync(cnt.ptr, 0, cnt.bytes, st));  // reused as the scatter cursor
    {
        b_scatter<<<grid, 256, 0, st>>>(pairs, np, off.as<unsigned long long>(), cnt.as<unsigned long long>(), wt, seed,
                                        packed.as<uint64_t>());
        ::hc::count_launch();
    }
    HC_CUDA_TRY(cudaGetLastError());

    // 4-5. sorted rows, duplicates dropped.
    HC_TRY(B.sort_rows(off.as<unsigned long long>(), (int32_t)n, packed.as<uint64_t>(), sorted.as<uint64_t>(), rel));
    DevBuf ndeg, maxdeg;
    HC_TRY(ndeg.ensure(sizeof(unsigned long long) * ((size_t)n + 1)));
    HC_TRY(maxdeg.ensure(sizeof(unsigned long long)));
    HC_CUDA_TRY(cudaMemsetAsync(maxdeg.ptr, 0, sizeof(unsigned long long), st));
    {
        b_dedup<<<grid, 256, 0, st>>>(off.as<unsigned long long>(), (int32_t)n, sorted.as<uint64_t>(),
                                      ndeg.as<unsigned long long>(), maxdeg.as<unsigned long long>());
        ::hc::count_launch();
    }
    HC_CUDA_TRY(cudaGetLastError());

    // 6. ranks by (degree desc, id desc).
    DevBuf keys, keys2, ids, order, rank, deg_new, noff;
    HC_TRY(keys.ensure(sizeof(uint64_t) * (size_t)n));
    HC_TRY(keys2.ensure(sizeof(uint64_t) * (size_t)n));
    HC_TRY(ids.ensure(sizeof(int32_t) * (size_t)n));
    HC_TRY(order.ensure(sizeof(int32_t) * (size_t)n));
    {
        b_rank_keys<<<grid, 256, 0, st>>>(ndeg.as<unsigned long long>(), (int32_t)n, maxdeg.as<unsigned long long>(),
                                          keys.as<uint64_t>(), ids.as<int32_t>());
        ::hc::count_launch();
    }
    {
        size_t bytes = 0;
        HC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                                    ids.as<int32_t>(), order.as<int32_t>(), (int)n, 0, 64, st));
        HC_TRY(B.temp.ensure(bytes));
        HC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(B.temp.ptr, bytes, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                                    ids.as<int32_t>(), order.as<int32_t>(), (int)n, 0, 64, st));
        ::hc::count_launch();
    }
    keys.release();
    keys2.release();
    ids.release();
    HC_TRY(rank.ensure(sizeof(int32_t) * (size_t)n));
    HC_TRY(deg_new.ensure(sizeof(unsigned long long) * ((size_t)n + 1)));
    HC_TRY(noff.ensure(sizeof(unsigned long long) * ((size_t)n + 1)));
    HC_CUDA_TRY(cudaMemsetAsync(deg_new.as<unsigned long long>() + n, 0, sizeof(unsigned long long), st));
    {
        b_rank<<<grid, 256, 0, st>>>(order.as<int32_t>(), (int32_t)n, ndeg.as<unsigned long long>(),
                                     rank.as<int32_t>(), deg_new.as<unsigned long long>());
        ::hc::count_launch();
    }
    HC_TRY(B.scan(deg_new.as<unsigned long long>(), noff.as<unsigned long long>(), n + 1));
    HC_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m = (int64_t)read1(noff.as<unsigned long long>() + n);
    order.release();
    deg_new.release();

    // 7. renamed rows in the new order (into `packed`), sorted (into `sorted`).
    {
        b_rename<<<grid, 256, 0, st>>>(off.as<unsigned long long>(), ndeg.as<unsigned long long>(), rank.as<int32_t>(),
                                       sorted.as<uint64_t>(), noff.as<unsigned long long>(), (int32_t)n,
                                       packed.as<uint64_t>());
        ::hc::count_launch();
    }
    HC_CUDA_TRY(cudaGetLastError());
    rank.release();
    ndeg.release();
    HC_TRY(B.sort_rows(noff.as<unsigned long long>(), (int32_t)n, packed.as<uint64_t>(), sorted.as<uint64_t>(), rel));
    rel.release();
    B.temp.release();

    // 8. neighbour and weight arrays (in `packed`, now free), int64 offsets (in `off`).
    int32_t *nbr = packed.as<int32_t>();
    uint32_t *w = wt != HC_W_NONE ? reinterpret_cast<uint32_t *>(nbr + m) : nullptr;
    { b_split<<<grid, 256, 0, st>>>(sorted.as<uint64_t>(), m, nbr, w); ::hc::count_launch(); }
    { b_to_i64<<<grid, 256, 0, st>>>(noff.as<unsigned long long>(), n + 1, off.as<int64_t>()); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    HC_CUDA_TRY(cudaStreamSynchronize(st));
    sorted.release();
    noff.release();
    cnt.release();
    return hc_graph_create(off.as<int64_t>(), nbr, w, wt, (int32_t)n, m, device, out);
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_graph_generate(hc_gen_kind kind, int32_t scale, int32_t edge_factor, uint64_t seed,
                                       hc_wtype wtype, int32_t device, hc_graph **out) {
    clear_error();
    if (!out || scale < 1 || scale > 30 || edge_factor < 1)
        return fail(HC_ERR_INVALID_ARG, "hc_graph_generate: bad scale %d / edge factor %d", scale, edge_factor);
    *out = nullptr;
    const int64_t np = (int64_t)edge_factor << scale;
    if (kind == HC_GEN_KRONECKER) return build_device(RmatPairs(scale, seed), scale, np, wtype, seed, device, out);
    if (kind == HC_GEN_UNIFORM) return build_device(UniformPairs{scale, seed}, scale, np, wtype, seed, device, out);
    return fail(HC_ERR_INVALID_ARG, "hc_graph_generate: unknown generator %d", (int)kind);
}

extern "C" hc_status hc_graph_get_csr(hc_graph *g, int64_t *index, int32_t *neighbors, void *weights) {
    clear_error();
    HC_TRY(activate(g));
    if (index) HC_TRY(copy_out(index, g->index.ptr, sizeof(int64_t) * ((size_t)g->N + 1), g->stream));
    if (neighbors) HC_TRY(copy_out(neighbors, g->nbr.ptr, sizeof(int32_t) * (size_t)g->M, g->stream));
    if (weights) {
        if (g->wtype == HC_W_NONE) return fail(HC_ERR_INVALID_ARG, "hc_graph_get_csr: graph has no weights");
        HC_TRY(copy_out(weights, g->wgt.ptr, 4 * (size_t)g->M, g->stream));
    }
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return HC_OK;
}

extern "C" hc_status hc_graph_pick_sources(hc_graph *g, int32_t count, int32_t *out) {
    clear_error();
    HC_TRY(activate(g));
    if (!out || count < 0) return fail(HC_ERR_INVALID_ARG, "hc_graph_pick_sources: bad arguments");
    std::vector<int64_t> idx((size_t)g->N + 1);
    HC_CUDA_TRY(cudaMemcpy(idx.data(), g->index.ptr, sizeof(int64_t) * idx.size(), cudaMemcpyDeviceToHost));
    const int32_t *nbr = g->nbr.as<int32_t>();
    // Degree-1 candidates read their one neighbour from the device.
    auto self_only = [&](int32_t v) { return read1(nbr + idx[v]) == v; };
    return pick_sources_impl(idx.data(), g->N, count, -1, out, self_only);
}
