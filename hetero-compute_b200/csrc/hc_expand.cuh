// Load-balanced expansion of a vertex queue over its CSR rows, shared by the
// top-down BFS and the SSSP relaxation.
//
// A warp takes 32 queue entries, scans their degrees and walks the combined
// edge range 32 edges at a time, so neighbour loads stay coalesced within a
// row whatever the degree mix.  Rows longer than kChunk edges are cut into
// (vertex, chunk) tasks that every warp of the grid shares after a barrier,
// which keeps hub rows from serialising on one warp.
#pragma once

#include "hc_device.cuh"

namespace hc {

constexpr int kChunk = 1024;

// Upper bound of the task list a queue can produce.
inline int64_t max_expand_tasks(int64_t m, int64_t n) { return 2 * (m / kChunk) + n / kChunk + 64; }

// fn(active, u, e) is called by all 32 lanes together (it may use warp
// collectives); `active` says whether lane's edge slot e of row u is real.
template <class EdgeFn>
__device__ __forceinline__ void expand_small(const int64_t *__restrict__ index, const int32_t *q, int nf,
                                             int2 *tasks, int *task_count, int gwarp, int nwarps,
                                             EdgeFn &fn) {
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
            if (deg > kChunk) {
                const int nt = (deg + kChunk - 1) / kChunk;
                const int t0 = atomicAdd(task_count, nt);
                for (int c = 0; c < nt; c++) tasks[t0 + c] = make_int2(u, c);
                deg = 0;
            }
        }
        int total;
        const int excl = warp_exclusive_scan(deg, &total);
        for (int k0 = 0; k0 < total; k0 += 32) {
            const int k = k0 + lane;
            int lo = 0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                const int c = __shfl_sync(kFull, excl, lo + s);
                if (c <= k) lo += s;
            }
            const int32_t uo = __shfl_sync(kFull, u, lo);
            const long long bo = __shfl_sync(kFull, beg, lo);
            const int off = k - __shfl_sync(kFull, excl, lo);
            fn(k < total, uo, (int64_t)(bo + off));
        }
    }
}

template <class EdgeFn>
__device__ __forceinline__ void expand_tasks(const int64_t *__restrict__ index, const int2 *tasks, int ntasks,
                                             int gwarp, int nwarps, EdgeFn &fn) {
    const int lane = threadIdx.x & 31;
    for (int t = gwarp; t < ntasks; t += nwarps) {
        const int2 tk = __ldcg(tasks + t);
        const int64_t rb = index[tk.x], re = index[tk.x + 1];
        const int64_t beg = rb + (int64_t)tk.y * kChunk;
        const int64_t end = min(re, beg + (int64_t)kChunk);
        for (int64_t e0 = beg; e0 < end; e0 += 32) {
            const int64_t e = e0 + lane;
            fn(e < end, tk.x, e);
        }
    }
}

// Appends `v` for every lane with `take` set to q[*len ...], one atomic per warp.
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

}  // namespace hc
