// Load-balanced expansion of a vertex queue over its CSR rows, shared by the
// top-down BFS and the SSSP relaxation.
//
// Rows of at most kSmallDeg edges are expanded warp-centrically: a warp takes
// 32 queue entries, scans their degrees and walks the combined edge range, so
// neighbour loads stay coalesced within a row whatever the degree mix.  Longer
// rows are cut into (vertex, chunk) tasks of kTaskEdges edges that every warp
// of the grid shares after a barrier, so hub rows and small frontiers of
// medium-degree vertices spread over the whole GPU.
//
// Each lane keeps kUnroll edges in flight: all neighbour loads of a round are
// issued, then all probes of the destination state, then the commits, which
// turns a chain of dependent memory round trips per edge into one per round.
//
// A visitor V provides
//   struct Item;                                   per-edge registers
//   void load(Item&, int32_t u, int64_t e)         neighbour (and weight) of slot e of row u
//   void probe(Item&)                              read destination state
//   void commit(Item (&)[kUnroll], const bool (&active)[kUnroll])
//                                                  update all items of a round; called by all
//                                                  32 lanes together (may use warp collectives)
#pragma once

#include "hc_device.cuh"

namespace hc {

constexpr int kSmallDeg = 32;
constexpr int kTaskEdges = 256;
constexpr int kUnroll = 4;

// Upper bound of the task list one queue can produce:
// sum over rows longer than kSmallDeg of ceil(deg / kTaskEdges).
inline int64_t max_expand_tasks(int64_t m, int64_t n) {
    (void)n;
    return m / kTaskEdges + m / (kSmallDeg + 1) + 64;
}

template <class V>
__device__ __forceinline__ void expand_small(const int64_t *__restrict__ index, const int32_t *q, int nf,
                                             int2 *tasks, int *task_count, int gwarp, int nwarps, V &vis) {
    const int lane = threadIdx.x & 31;
    for (int base = gwarp * 32; base < nf; base += nwarps * 32) {
        const int i = base + lane;
        int32_t u = -1;
        long long beg = 0;
        int deg = 0;
        if (i < nf) {
            u = ld_cg(q + i);
            beg = index[u];
            deg = (int)(index[u + 1] - beg);
            if (deg > kSmallDeg) {
                const int nt = (deg + kTaskEdges - 1) / kTaskEdges;
                const int t0 = atomicAdd(task_count, nt);
                for (int c = 0; c < nt; c++) tasks[t0 + c] = make_int2(u, c);
                deg = 0;
            }
        }
        int total;
        const int excl = warp_exclusive_scan(deg, &total);
        for (int k0 = 0; k0 < total; k0 += 32 * kUnroll) {
            typename V::Item it[kUnroll];
            bool act[kUnroll];
#pragma unroll
            for (int j = 0; j < kUnroll; j++) {
                const int k = k0 + 32 * j + lane;
                int lo = 0;
#pragma unroll
                for (int s = 16; s > 0; s >>= 1) {
                    const int c = __shfl_sync(kFull, excl, lo + s);
                    if (c <= k) lo += s;
                }
                const int32_t uo = __shfl_sync(kFull, u, lo);
                const long long bo = __shfl_sync(kFull, beg, lo);
                const int off = k - __shfl_sync(kFull, excl, lo);
                act[j] = k < total;
                if (act[j]) vis.load(it[j], uo, (int64_t)(bo + off));
            }
#pragma unroll
            for (int j = 0; j < kUnroll; j++)
                if (act[j]) vis.probe(it[j]);
            vis.commit(it, act);
        }
    }
}

template <class V>
__device__ __forceinline__ void expand_tasks(const int64_t *__restrict__ index, const int2 *tasks, int ntasks,
                                             int gwarp, int nwarps, V &vis) {
    const int lane = threadIdx.x & 31;
    for (int t = gwarp; t < ntasks; t += nwarps) {
        const int2 tk = __ldcg(tasks + t);
        const int64_t rb = index[tk.x], re = index[tk.x + 1];
        const int64_t beg = rb + (int64_t)tk.y * kTaskEdges;
        const int64_t end = min(re, beg + (int64_t)kTaskEdges);
        for (int64_t e0 = beg; e0 < end; e0 += 32 * kUnroll) {
            typename V::Item it[kUnroll];
            bool act[kUnroll];
#pragma unroll
            for (int j = 0; j < kUnroll; j++) {
                const int64_t e = e0 + 32 * j + lane;
                act[j] = e < end;
                if (act[j]) vis.load(it[j], tk.x, e);
            }
#pragma unroll
            for (int j = 0; j < kUnroll; j++)
                if (act[j]) vis.probe(it[j]);
            vis.commit(it, act);
        }
    }
}

// Appends `v` for every lane with `take` set to q[*len ...], one atomic per warp.
// Word of a frontier bitmap that holds vertex u's bit: from a shared-memory
// copy of the bitmap's first hub_v / 32 words when u is in it, else from the
// bitmap in global memory.  Both loads always issue (no branch, so the probes
// of a round stay in flight); a copied vertex points its global load at word
// 0, one line for the whole warp.  u < 0 (no edge) reads as 0.  On
// degree-sorted graphs the copied prefix holds the hubs most edges point at.
__device__ __forceinline__ uint32_t frontier_word(const uint32_t *s_fb, int hub_v, const uint32_t *fb, int32_t u) {
    const bool hub = u >= 0 && u < hub_v;
    const uint32_t sw = s_fb[hub ? (u >> 5) : 0];
    const uint32_t gw = u >= 0 ? __ldcg(fb + (hub ? 0 : (u >> 5))) : 0u;
    return hub ? sw : gw;
}

__device__ __forceinline__ void warp_append(bool take, int32_t v, int32_t *q, int *len) {
    const unsigned bal = __ballot_sync(kFull, take);
    if (!bal) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(bal) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(len, __popc(bal));
    base = __shfl_sync(kFull, base, leader);
    if (take) q[base + __popc(bal & ((1u << lane) - 1u))] = v;
}

// Appends up to kUnroll values per lane with a single atomic per warp.
__device__ __forceinline__ void warp_append_n(const bool (&take)[kUnroll], const int32_t (&v)[kUnroll], int32_t *q,
                                              int *len) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    unsigned bal[kUnroll];
    int total = 0;
#pragma unroll
    for (int j = 0; j < kUnroll; j++) {
        bal[j] = __ballot_sync(kFull, take[j]);
        total += __popc(bal[j]);
    }
    if (total == 0) return;
    int base = 0;
    if (lane == 0) base = atomicAdd(len, total);
    base = __shfl_sync(kFull, base, 0);
#pragma unroll
    for (int j = 0; j < kUnroll; j++) {
        if (take[j]) q[base + __popc(bal[j] & lt)] = v[j];
        base += __popc(bal[j]);
    }
}

}  // namespace hc
