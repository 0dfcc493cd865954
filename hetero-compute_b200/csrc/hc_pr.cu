// Pull PageRank: forward, adjoint and multi-column (personalised) forms.
//
// Reference path: pr_pull_gpu (src/kernels/gpu/pr.cuh:42-118) with the
// in-place epochs of src/kernels/gpu/pr.cuh:140-318: score[v] = (1-d)/N +
// d * sum_u score[u]/deg[u], reading an 8-byte wnode_t and an 8-byte int64
// degree per edge.  Here each iteration is a Jacobi pull over a gathered
// vector that already carries the 1/deg factor (4-byte neighbour stream +
// 4-byte gather), with the L1 / per-vertex residual reduced in the same pass.
//
// Work plan (built once per graph from the row offsets):
//   stream groups  32 consecutive rows with <= kStreamEdges edges in total;
//                  one warp streams the whole edge range coalesced and reduces
//                  it segment by segment (CSR-stream, Greathouse & Daga 2014)
//   long rows      one warp per row, 128-bit neighbour loads
//   hub rows       > kHubEdges edges, cut into kHubChunk-edge chunks; each
//                  chunk's warp writes a partial, the last one to finish sums
//                  the partials in chunk order (deterministic) and finalises
// Vertices without edges keep (1-d) t_v, written once before the iterations.
#include <algorithm>
#include <cmath>
#include <vector>

#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr int kPrThreads = 256;
constexpr int kMaxIterSlots = 4096;

struct IterState {
    double l1[kMaxIterSlots];
    int changed[kMaxIterSlots];
    unsigned blocks_done;
    int done;
    int iters;
    int pad;
};

// One pull sweep: out[v] = base_v + d * rs_v * sum_{e in row v} ew_e * gin[nbr_e].
struct SweepArgs {
    const int64_t *index;
    const int32_t *nbr;
    const float *ew;        // per-slot edge weight (kEW)
    const float *gin;       // gathered vector
    const float *xin;       // previous iterate (residual)
    const float *basev;     // per-vertex base (kBaseVec), already scaled by (1-d)
    float base_scalar;
    float d;
    const float *rs;        // per-row scale (kRS)
    const float *ps;        // gather-out scale (kPS)
    float *xout;
    float *gout;            // gather vector for the next sweep (kPS) -- else == xout
    float *partials;
    unsigned *hub_count;
    IterState *st;
    int it;
    float omega;            // Chebyshev weight of this iteration (1: plain Jacobi)
    float tol_l1, eps;
    int max_iters;
    int32_t n_active;
};

template <bool kEW, bool kRS, bool kPS, bool kBaseVec, bool kCG = false>
__device__ __forceinline__ void finish_row(const SweepArgs &a, int32_t r, float sum, float &l1, int &chg) {
    if constexpr (kCG) {
        // Conjugate-gradient product (gin = p): xout = (S p)_r, and
        // p_r q_r with q = s p - d S p summed where the residual goes.
        const float pr = a.gin[r];
        const float rsr = a.rs[r];
        const float sr = rsr > 0.f ? 1.0f / rsr : 0.f;
        a.xout[r] = sum;
        l1 += pr * (sr * pr - a.d * sum);
        return;
    }
    const float base = kBaseVec ? a.basev[r] : a.base_scalar;
    const float scale = kRS ? a.rs[r] : 1.0f;
    float nv = base + a.d * (scale * sum);
    const float ov = a.xin[r];
    // The residual |J(x_k) - x_k| of the fixed-point equation: the change of
    // a plain Jacobi sweep, and the stopping rule of both iterations.
    const float dl = fabsf(nv - ov);
    // Chebyshev semi-iteration: x_{k+1} = omega (J(x_k) - x_{k-1}) + x_{k-1};
    // x_{k-1} is what the output buffer still holds.
    if (a.omega != 1.0f) {
        const float prev = a.xout[r];
        nv = a.omega * (nv - prev) + prev;
    }
    a.xout[r] = nv;
    if (kPS) a.gout[r] = nv * a.ps[r];
    l1 += dl;
    chg += dl > a.eps;
}

template <bool kEW>
__device__ __forceinline__ float edge_val(const SweepArgs &a, int64_t e) {
    const float g = __ldg(a.gin + a.nbr[e]);
    return kEW ? g * a.ew[e] : g;
}

template <bool kEW, bool kRS, bool kPS, bool kBaseVec, bool kCG = false>
__global__ void __launch_bounds__(kPrThreads) pr_sweep(SweepArgs a, PrPlanDev plan) {
    __shared__ float s_acc[kPrThreads / 32][32];
    __shared__ double s_l1[32];
    __shared__ int s_chg[32];
    __shared__ int s_last;
    if (*(volatile int *)&a.st->done) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    float l1 = 0.f;
    int chg = 0;
    const int total_items = plan.n_tasks + plan.n_long + plan.n_stream;

    for (int item = gwarp; item < total_items; item += nwarps) {
        if (item < plan.n_tasks) {
            // Chunk of a hub row.
            const int2 tk = plan.tasks[item];
            const HubInfo h = plan.hubs[tk.x];
            const int64_t rb = a.index[h.row], re = a.index[h.row + 1];
            const int64_t b = rb + (int64_t)tk.y * kHubChunk;
            const int64_t e = min(re, b + (int64_t)kHubChunk);
            // Four independent partial sums keep four gathers in flight.
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
            int64_t i = b + lane;
            for (; i + 96 < e; i += 128) {
                s0 += edge_val<kEW>(a, i);
                s1 += edge_val<kEW>(a, i + 32);
                s2 += edge_val<kEW>(a, i + 64);
                s3 += edge_val<kEW>(a, i + 96);
            }
            for (; i < e; i += 32) s0 += edge_val<kEW>(a, i);
            float s = warp_sum((s0 + s1) + (s2 + s3));
            int last = 0;
            if (lane == 0) {
                a.partials[h.first + tk.y] = s;
                __threadfence();
                last = atomicAdd(a.hub_count + tk.x, 1u) == (unsigned)(h.nchunks - 1);
            }
            last = __shfl_sync(kFull, last, 0);
            if (last) {
                __threadfence();
                float t = 0.f;
                for (int c = lane; c < h.nchunks; c += 32) t += __ldcg(a.partials + h.first + c);
                t = warp_sum(t);
                if (lane == 0) {
                    a.hub_count[tk.x] = 0;
                    finish_row<kEW, kRS, kPS, kBaseVec, kCG>(a, h.row, t, l1, chg);
                }
            }
        } else if (item < plan.n_tasks + plan.n_long) {
            const int32_t r = plan.longrows[item - plan.n_tasks];
            const int64_t b = a.index[r], e = a.index[r + 1];
            float s = 0.f;
            // Scalar head up to a 16-byte boundary, then 128-bit neighbour loads.
            const int64_t ab = min(e, (b + 3) & ~(int64_t)3);
            if (b + lane < ab) s += edge_val<kEW>(a, b + lane);
            for (int64_t i = ab + 4 * lane; i + 3 < e; i += 128) {
                const int4 v4 = *reinterpret_cast<const int4 *>(a.nbr + i);
                if (kEW) {
                    const float4 w4 = *reinterpret_cast<const float4 *>(a.ew + i);
                    s += __ldg(a.gin + v4.x) * w4.x + __ldg(a.gin + v4.y) * w4.y +
                         __ldg(a.gin + v4.z) * w4.z + __ldg(a.gin + v4.w) * w4.w;
                } else {
                    s += (__ldg(a.gin + v4.x) + __ldg(a.gin + v4.y)) + (__ldg(a.gin + v4.z) + __ldg(a.gin + v4.w));
                }
            }
            const int64_t tail = ab + ((e - ab) & ~(int64_t)3);
            if (tail + lane < e) s += edge_val<kEW>(a, tail + lane);
            s = warp_sum(s);
            if (lane == 0) finish_row<kEW, kRS, kPS, kBaseVec, kCG>(a, r, s, l1, chg);
        } else {
            // Stream group: rows r0 .. r0+31 (clipped to n_active).
            const int32_t r0 = plan.stream[item - plan.n_tasks - plan.n_long] * 32;
            const int32_t r = r0 + lane;
            const int32_t rc = min(r, a.n_active);
            const int64_t s0 = a.index[r0];
            const int32_t rel = (int32_t)(a.index[rc] - s0);  // start of this lane's row
            const int32_t gend = (int32_t)(a.index[min(r0 + 32, a.n_active)] - s0);
            s_acc[wib][lane] = 0.f;
            __syncwarp();
            // Four 32-edge chunks per pass: their loads and gathers are issued
            // together, then each chunk is summed by its segmented scan in the
            // same order as one chunk at a time.
            for (int k0 = 0; k0 < gend; k0 += 128) {
                float vals[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int k = k0 + 32 * j + lane;
                    vals[j] = k < gend ? edge_val<kEW>(a, s0 + k) : 0.f;
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int kb = k0 + 32 * j;
                    if (kb >= gend) break;
                    const int k = kb + lane;
                    const bool act = k < gend;
                    int lo = 0;
#pragma unroll
                    for (int st = 16; st > 0; st >>= 1) {
                        const int c = __shfl_sync(kFull, rel, lo + st);
                        if (c <= k) lo += st;
                    }
                    int owner = act ? lo : 32;
                    float v = vals[j];
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const float y = __shfl_up_sync(kFull, v, o);
                        const int ow = __shfl_up_sync(kFull, owner, o);
                        if (lane >= o && ow == owner) v += y;
                    }
                    const int next_owner = __shfl_down_sync(kFull, owner, 1);
                    const bool tail = (lane == 31) || next_owner != owner;
                    if (act && tail) s_acc[wib][owner] += v;
                    __syncwarp();
                }
            }
            if (r < a.n_active) finish_row<kEW, kRS, kPS, kBaseVec, kCG>(a, r, s_acc[wib][lane], l1, chg);
            __syncwarp();
        }
    }

    // Residual reduction; the last block to finish decides convergence.
    double dl1 = warp_sum((double)l1);
    int dchg = warp_sum(chg);
    if (lane == 0) {
        s_l1[wib] = dl1;
        s_chg[wib] = dchg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        int c = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
            t += s_l1[i];
            c += s_chg[i];
        }
        const int slot = a.it % kMaxIterSlots;
        if (t != 0.0) atomicAdd(&a.st->l1[slot], t);
        if (c) atomicAdd(&a.st->changed[slot], c);
        __threadfence();
        s_last = atomicAdd(&a.st->blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        const int slot = a.it % kMaxIterSlots;
        const double tl1 = *(volatile double *)&a.st->l1[slot];
        const int tch = *(volatile int *)&a.st->changed[slot];
        // eps >= 3e38 marks the per-vertex rule as unused.
        const bool conv = (a.tol_l1 > 0.f && tl1 < (double)a.tol_l1) || (a.eps < 3e38f && tch == 0);
        a.st->iters = a.it + 1;
        a.st->blocks_done = 0;
        // Clear the slot the next sweep will use.
        const int ns = (a.it + 1) % kMaxIterSlots;
        a.st->l1[ns] = 0.0;
        a.st->changed[ns] = 0;
        if (conv || a.it + 1 >= a.max_iters) a.st->done = conv ? 1 : 2;
    }
}

// x <- (1-d) t (or (1-d)/N) for every vertex; gather vector g <- x * ps.
// Rows that may have edges start from x0_scale * (x0v or x0_scalar).
__global__ void pr_init(int32_t n, const float *basev, float base_scalar, float x0_scalar, const float *x0v,
                        float x0_scale, const float *ps, float *x, float *g, float *x2, float *g2, int32_t n_active) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float base = basev ? basev[v] : base_scalar;
        // Vertices without edges sit at their base from the start; the rest
        // start from the initial guess.
        const float x0 = v >= n_active ? base : x0_scale * (x0v ? x0v[v] : x0_scalar);
        x[v] = x0;
        x2[v] = x0;
        if (g) {
            const float gv = ps ? x0 * ps[v] : x0;
            g[v] = gv;
            g2[v] = gv;
        }
    }
}

__global__ void sum_abs(const float *v, int32_t n, double *out) {
    __shared__ double s_red[32];
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += fabs((double)v[i]);
    s = block_sum(s, s_red);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(out, s);
}

__global__ void scale_vec(const float *in, float s, float *out, size_t n) {
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x)
        out[v] = s * in[v];
}

// dL/dw_uk = (d x_u / s_u) (lambda_k - sum_j W_uj lambda_j), slot order of
// row u, and at the fixed point sum_j W_uj lambda_j = (lambda_u - c_u) / d, so one pass:
// dL/dw_uk = (x_u / s_u) (d lambda_k - lambda_u + c_u).
// Work items are the row plan's: hub chunks and long rows (one warp, one row)
// and stream groups (32 rows, one warp walks their edges 32 at a time and
// each lane finds its edge's row among the group's offsets).
__global__ void __launch_bounds__(kPrThreads) pr_edge_grad(PrPlanDev plan, const int64_t *index, const int32_t *nbr,
                                                           const float *rs, const float *x, const float *lam,
                                                           const float *c, float d, int32_t n_active, float *grad) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int total = plan.n_tasks + plan.n_long + plan.n_stream;
    for (int item = gwarp; item < total; item += nwarps) {
        if (item < plan.n_tasks + plan.n_long) {
            int32_t u;
            int64_t b, e;
            if (item < plan.n_tasks) {
                const int2 tk = plan.tasks[item];
                u = plan.hubs[tk.x].row;
                const int64_t rb = index[u], re = index[u + 1];
                b = rb + (int64_t)tk.y * kHubChunk;
                e = min(re, b + (int64_t)kHubChunk);
            } else {
                u = plan.longrows[item - plan.n_tasks];
                b = index[u];
                e = index[u + 1];
            }
            const float coef = x[u] * rs[u];
            const float off = lam[u] - c[u];
            for (int64_t i = b + lane; i < e; i += 32) grad[i] = coef * (d * __ldg(lam + nbr[i]) - off);
        } else {
            const int32_t r0 = plan.stream[item - plan.n_tasks - plan.n_long] * 32;
            const int32_t r = r0 + lane;
            const int32_t rc = min(r, n_active);
            const int64_t s0 = index[r0];
            const int32_t rel = (int32_t)(index[rc] - s0);
            const int32_t gend = (int32_t)(index[min(r0 + 32, n_active)] - s0);
            const float coef = r < n_active ? x[r] * rs[r] : 0.f;
            const float off = r < n_active ? lam[r] - c[r] : 0.f;
            for (int k0 = 0; k0 < gend; k0 += 32) {
                const int k = k0 + lane;
                int lo = 0;
#pragma unroll
                for (int st = 16; st > 0; st >>= 1) {
                    const int cc = __shfl_sync(kFull, rel, lo + st);
                    if (cc <= k) lo += st;
                }
                const float cf = __shfl_sync(kFull, coef, lo);
                const float of = __shfl_sync(kFull, off, lo);
                if (k < gend) grad[s0 + k] = cf * (d * __ldg(lam + nbr[s0 + k]) - of);
            }
        }
    }
}

// ---------------------------------------------------------------- SpMM form
// K columns per vertex, vertex-major [N][K]; warp per row, lane c handles
// columns c, c+32, ...; hub rows are chunked like the single-column plan.
struct SpmmArgs {
    const int64_t *index;
    const int32_t *nbr;
    const float *ew;
    const float *gin;        // [N][K], already divided by deg (unweighted)
    const float *xin;
    const float *basev;      // [N][K] dense base, or null with seeds
    const int32_t *seed_off; // sparse teleport: column c has seeds seed_idx[seed_off[c]..seed_off[c+1])
    const int32_t *seed_idx;
    float d;
    const float *ps;         // per-row gather scale
    float *xout, *gout;
    float *partials;         // [chunks][K]
    unsigned *hub_count;
    double *col_l1;          // [K] accumulators for this sweep
    const int32_t *col_map;  // packed column -> seed-list column (null: identity)
    int K;                   // columns in the packed layout
    int32_t n_active;
};

__device__ __forceinline__ float spmm_base(const SpmmArgs &a, int32_t r, int c, float one_minus_d) {
    if (a.basev) return a.basev[(size_t)r * a.K + c];
    // Uniform over the seed set of column c.
    const int cc = a.col_map ? a.col_map[c] : c;
    const int32_t b = a.seed_off[cc], e = a.seed_off[cc + 1];
    for (int32_t i = b; i < e; i++)
        if (a.seed_idx[i] == r) return one_minus_d / (float)(e - b);
    return 0.f;
}

template <int kCols>
__global__ void __launch_bounds__(kPrThreads) spmm_sweep(SpmmArgs a, PrPlanDev plan, const uint8_t *is_seed) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int K = a.K;
    const float omd = 1.0f - a.d;
    float l1[kCols];
#pragma unroll
    for (int j = 0; j < kCols; j++) l1[j] = 0.f;
    // Every row with edges is its own item here (long rows and stream rows
    // alike); hub rows are chunked.
    const int n_rows = a.n_active;
    const int total = plan.n_tasks + n_rows;
    auto finish = [&](int32_t r, float *acc) {
        const float pscale = a.ps ? a.ps[r] : 1.0f;
        const bool seed = is_seed ? is_seed[r] != 0 : true;
#pragma unroll
        for (int j = 0; j < kCols; j++) {
            const int c = lane + 32 * j;
            if (c < K) {
                const size_t o = (size_t)r * K + c;
                const float base = seed ? spmm_base(a, r, c, omd) : 0.f;
                const float nv = base + a.d * acc[j];
                const float ov = a.xin[o];
                a.xout[o] = nv;
                if (a.gout != a.xout) a.gout[o] = nv * pscale;
                l1[j] += fabsf(nv - ov);
            }
        }
    };
    for (int item = gwarp; item < total; item += nwarps) {
        float acc[kCols];
#pragma unroll
        for (int j = 0; j < kCols; j++) acc[j] = 0.f;
        if (item < plan.n_tasks) {
            const int2 tk = plan.tasks[item];
            const HubInfo h = plan.hubs[tk.x];
            const int64_t rb = a.index[h.row], re = a.index[h.row + 1];
            const int64_t b = rb + (int64_t)tk.y * kHubChunk;
            const int64_t e = min(re, b + (int64_t)kHubChunk);
            for (int64_t i = b; i < e; i++) {
                const int32_t u = a.nbr[i];
                const float wv = a.ew ? a.ew[i] : 1.0f;
                const float *gu = a.gin + (size_t)u * K;
#pragma unroll
                for (int j = 0; j < kCols; j++) {
                    const int c = lane + 32 * j;
                    if (c < K) acc[j] += wv * __ldg(gu + c);
                }
            }
#pragma unroll
            for (int j = 0; j < kCols; j++) {
                const int c = lane + 32 * j;
                if (c < K) a.partials[(size_t)(h.first + tk.y) * K + c] = acc[j];
            }
            __syncwarp();
            int last = 0;
            if (lane == 0) {
                __threadfence();
                last = atomicAdd(a.hub_count + tk.x, 1u) == (unsigned)(h.nchunks - 1);
            }
            last = __shfl_sync(kFull, last, 0);
            if (last) {
                __threadfence();
#pragma unroll
                for (int j = 0; j < kCols; j++) acc[j] = 0.f;
                for (int ch = 0; ch < h.nchunks; ch++) {
#pragma unroll
                    for (int j = 0; j < kCols; j++) {
                        const int c = lane + 32 * j;
                        if (c < K) acc[j] += __ldcg(a.partials + (size_t)(h.first + ch) * K + c);
                    }
                }
                if (lane == 0) a.hub_count[tk.x] = 0;
                finish(h.row, acc);
            }
        } else {
            const int32_t r = item - plan.n_tasks;
            const int64_t b = a.index[r], e = a.index[r + 1];
            if (e - b > kHubEdges) continue;  // handled as chunks
            for (int64_t i = b; i < e; i++) {
                const int32_t u = a.nbr[i];
                const float wv = a.ew ? a.ew[i] : 1.0f;
                const float *gu = a.gin + (size_t)u * K;
#pragma unroll
                for (int j = 0; j < kCols; j++) {
                    const int c = lane + 32 * j;
                    if (c < K) acc[j] += wv * __ldg(gu + c);
                }
            }
            finish(r, acc);
        }
    }
#pragma unroll
    for (int j = 0; j < kCols; j++) {
        const int c = lane + 32 * j;
        if (c < K && l1[j] != 0.f) atomicAdd(a.col_l1 + c, (double)l1[j]);
    }
}

// Start: each column's teleport t (base / (1-d)), which has the fixed
// point's mass; vertices without edges sit at their base (1-d) t from the start.
__global__ void spmm_init(int32_t n, int K, const float *basev, const int32_t *seed_off, const int32_t *seed_idx,
                          const uint8_t *is_seed, float d, const float *ps, float *x, float *g, float *x2, float *g2,
                          int32_t n_active) {
    const size_t total = (size_t)n * K;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int32_t v = (int32_t)(i / K);
        const int c = (int)(i % K);
        float base = 0.f;
        if (basev) {
            base = basev[i];
        } else if (is_seed[v]) {
            const int32_t b = seed_off[c], e = seed_off[c + 1];
            for (int32_t j = b; j < e; j++)
                if (seed_idx[j] == v) base = (1.0f - d) / (float)(e - b);
        }
        const float t = v < n_active ? base / (1.0f - d) : base;
        x[i] = t;
        x2[i] = t;
        const float gv = ps ? t * ps[v] : t;
        g[i] = gv;
        g2[i] = gv;
    }
}

// Repacks the live columns of x ([n][kw]) into xo ([n][nkw], gather copy go =
// xo * ps when go is set); a column with newpos < 0 has converged and goes to
// its place col_map[c] in out ([n][K0]).  Rows stay contiguous on both sides.
__global__ void spmm_repack(int32_t n, int kw, const float *x, const int32_t *newpos, const int32_t *col_map,
                            int K0, float *out, int nkw, float *xo, float *go, const float *ps) {
    const size_t total = (size_t)n * kw;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int32_t v = (int32_t)(i / kw);
        const int c = (int)(i % kw);
        const float val = x[i];
        const int np = newpos[c];
        if (np < 0) {
            out[(size_t)v * K0 + col_map[c]] = val;
        } else {
            xo[(size_t)v * nkw + np] = val;
            if (go) go[(size_t)v * nkw + np] = ps ? val * ps[v] : val;
        }
    }
}

// One packed column c (width kw) as a plain vector (and its gather copy).
__global__ void spmm_take_column(int32_t n, int kw, int c, const float *x, const float *ps, float *x0, float *x1,
                                 float *g0, float *g1) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float val = x[(size_t)v * kw + c];
        x0[v] = val;
        x1[v] = val;
        if (g0) {
            const float gv = ps ? val * ps[v] : val;
            g0[v] = gv;
            g1[v] = gv;
        }
    }
}

// base[v] = (1-d) / |seeds| on the seeds of one column (base zeroed before).
__global__ void spmm_column_base(const int32_t *seed_idx, int32_t b, int32_t e, float one_minus_d, float *base) {
    for (int i = b + blockIdx.x * blockDim.x + threadIdx.x; i < e; i += gridDim.x * blockDim.x)
        base[seed_idx[i]] = one_minus_d / (float)(e - b);
}

__global__ void spmm_put_column(int32_t n, const float *x, int K0, int oc, float *out) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        out[(size_t)v * K0 + oc] = x[v];
}

__global__ void mark_seeds(const int32_t *seed_idx, int32_t nseeds, uint8_t *is_seed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nseeds; i += gridDim.x * blockDim.x)
        is_seed[seed_idx[i]] = 1;
}

__global__ void spmm_residual(const double *col_l1, int K, float tol, int *done_cols) {
    int c = 0;
    for (int i = threadIdx.x; i < K; i += blockDim.x) c += col_l1[i] < (double)tol;
    c = warp_sum(c);
    __shared__ int s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += s[i];
        *done_cols = t;
    }
}

}  // namespace

// ------------------------------------------------------------------- plan

hc_status ensure_plan(hc_graph *g) {
    if (g->pr_plan.ptr) return HC_OK;
    const int32_t na = g->n_active;
    std::vector<int64_t> idx((size_t)na + 1);
    HC_CUDA_TRY(cudaMemcpy(idx.data(), g->index.as<int64_t>(), sizeof(int64_t) * ((size_t)na + 1),
                           cudaMemcpyDeviceToHost));
    std::vector<int32_t> stream, longrows;
    std::vector<int2> tasks;
    std::vector<HubInfo> hubs;
    int32_t partial_slots = 0;
    const int32_t ngroups = (na + 31) / 32;
    for (int32_t gid = 0; gid < ngroups; gid++) {
        const int32_t r0 = gid * 32, r1 = std::min(r0 + 32, na);
        const int64_t tot = idx[r1] - idx[r0];
        if (tot <= kStreamEdges) {
            stream.push_back(gid);
            continue;
        }
        for (int32_t r = r0; r < r1; r++) {
            const int64_t d = idx[r + 1] - idx[r];
            if (d > kHubEdges) {
                HubInfo h{r, partial_slots, (int32_t)((d + kHubChunk - 1) / kHubChunk), 0};
                for (int c = 0; c < h.nchunks; c++) tasks.push_back(make_int2((int)hubs.size(), c));
                partial_slots += h.nchunks;
                hubs.push_back(h);
            } else {
                longrows.push_back(r);
            }
        }
    }
    const size_t b_hdr = 256;
    const size_t b_stream = (stream.size() * 4 + 255) / 256 * 256;
    const size_t b_long = (longrows.size() * 4 + 255) / 256 * 256;
    const size_t b_tasks = (tasks.size() * sizeof(int2) + 255) / 256 * 256;
    const size_t b_hubs = (hubs.size() * sizeof(HubInfo) + 255) / 256 * 256;
    HC_TRY(g->pr_plan.ensure(b_hdr + b_stream + b_long + b_tasks + b_hubs + 256));
    char *p = g->pr_plan.as<char>() + b_hdr;
    PrPlanDev v{};
    v.n_stream = (int)stream.size();
    v.n_long = (int)longrows.size();
    v.n_tasks = (int)tasks.size();
    v.n_hub = (int)hubs.size();
    v.stream = (const int32_t *)p;
    if (!stream.empty()) HC_CUDA_TRY(cudaMemcpy(p, stream.data(), stream.size() * 4, cudaMemcpyHostToDevice));
    p += b_stream;
    v.longrows = (const int32_t *)p;
    if (!longrows.empty()) HC_CUDA_TRY(cudaMemcpy(p, longrows.data(), longrows.size() * 4, cudaMemcpyHostToDevice));
    p += b_long;
    v.tasks = (const int2 *)p;
    if (!tasks.empty()) HC_CUDA_TRY(cudaMemcpy(p, tasks.data(), tasks.size() * sizeof(int2), cudaMemcpyHostToDevice));
    p += b_tasks;
    v.hubs = (const HubInfo *)p;
    if (!hubs.empty()) HC_CUDA_TRY(cudaMemcpy(p, hubs.data(), hubs.size() * sizeof(HubInfo), cudaMemcpyHostToDevice));
    g->pr_view = v;
    g->pr_partial_slots = partial_slots;
    return HC_OK;
}

namespace {

PrPlanDev plan_view(hc_graph *g, int *partial_slots) {
    *partial_slots = g->pr_partial_slots;
    return g->pr_view;
}

template <bool kEW, bool kRS, bool kPS, bool kBaseVec, bool kCG = false>
hc_status launch_sweep(hc_graph *g, const SweepArgs &a, const PrPlanDev &plan) {
    static int bps = 0;
    if (bps == 0) {
        HC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, pr_sweep<kEW, kRS, kPS, kBaseVec, kCG>,
                                                                  kPrThreads, 0));
        bps = std::max(bps, 1);
    }
    { pr_sweep<kEW, kRS, kPS, kBaseVec, kCG><<<g->sm_count * bps, kPrThreads, 0, g->stream>>>(a, plan); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    return HC_OK;
}

using SweepFn = hc_status (*)(hc_graph *, const SweepArgs &, const PrPlanDev &);

SweepFn pick_sweep(bool ew, bool rs, bool ps, bool basev) {
    const int key = (ew ? 8 : 0) | (rs ? 4 : 0) | (ps ? 2 : 0) | (basev ? 1 : 0);
    switch (key) {
        case 0: return launch_sweep<false, false, false, false>;
        case 1: return launch_sweep<false, false, false, true>;
        case 2: return launch_sweep<false, false, true, false>;
        case 3: return launch_sweep<false, false, true, true>;
        case 4: return launch_sweep<false, true, false, false>;
        case 5: return launch_sweep<false, true, false, true>;
        case 8: return launch_sweep<true, false, false, false>;
        case 9: return launch_sweep<true, false, false, true>;
        case 12: return launch_sweep<true, true, false, false>;
        case 13: return launch_sweep<true, true, false, true>;
        default: return nullptr;
    }
}

// Runs sweeps until the device marks the state done.  Launches are queued in
// rounds of kRound and the host checks the done flag once per round; sweeps
// queued after convergence return immediately.
struct SolveResult {
    int iters;
    int done;
    double l1;
    int changed;
    float ms;
};

// Sweeps until converged.  cheb_rho > 0: Chebyshev semi-iteration for a
// Jacobi operator whose spectrum lies in [-cheb_rho, cheb_rho] (a reversible
// walk scaled by d): weights omega_1 = 1, omega_2 = 1 / (1 - rho^2 / 2),
// omega_{k+1} = 1 / (1 - rho^2 omega_k / 4) (Golub and Varga, 1961).
hc_status run_solve(hc_graph *g, SweepArgs a, const PrPlanDev &plan, SweepFn fn, float *x[2], float *gv[2],
                    bool separate_g, SolveResult *res, float cheb_rho = 0.f) {
    IterState *st = reinterpret_cast<IterState *>(g->ws_ctl.ptr);
    HC_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(IterState), g->stream));
    HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    constexpr int kRound = 4;
    int host_done = 0;
    struct Tail {
        int done, iters;
    };
    HC_TRY(g->pinned.ensure(64));
    volatile Tail *pt = g->pinned.as<Tail>();
    const double rho2 = (double)cheb_rho * cheb_rho;
    double omega = 1.0;
    for (int it = 0; it < a.max_iters && !host_done;) {
        for (int k = 0; k < kRound && it < a.max_iters; k++, it++) {
            a.it = it;
            if (cheb_rho > 0.f) omega = it == 0 ? 1.0 : it == 1 ? 1.0 / (1.0 - rho2 / 2.0) : 1.0 / (1.0 - rho2 * omega / 4.0);
            a.omega = (float)omega;
            a.gin = separate_g ? gv[it & 1] : x[it & 1];
            a.xin = x[it & 1];
            a.xout = x[(it + 1) & 1];
            a.gout = separate_g ? gv[(it + 1) & 1] : a.xout;
            HC_TRY(fn(g, a, plan));
        }
        HC_CUDA_TRY(cudaMemcpyAsync((void *)pt, &st->done, sizeof(Tail), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        host_done = pt->done;
    }
    HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    Tail t;
    HC_CUDA_TRY(cudaMemcpy(&t, &st->done, sizeof(Tail), cudaMemcpyDeviceToHost));
    res->iters = t.iters;
    res->done = t.done;
    const int slot = (t.iters - 1) % kMaxIterSlots;
    double l1 = 0;
    int chg = 0;
    if (t.iters > 0) {
        HC_CUDA_TRY(cudaMemcpy(&l1, &st->l1[slot], sizeof(double), cudaMemcpyDeviceToHost));
        HC_CUDA_TRY(cudaMemcpy(&chg, &st->changed[slot], sizeof(int), cudaMemcpyDeviceToHost));
    }
    res->l1 = l1;
    res->changed = chg;
    HC_CUDA_TRY(cudaEventElapsedTime(&res->ms, g->ev_start, g->ev_stop));
    return HC_OK;
}

// ------------------------------------------------- adjoint by conjugate gradients
// For a reversible walk (symmetric weights S, weighted degrees s, D = diag(s))
// the adjoint equation lambda = c + d D^-1 S lambda is, multiplied by D, the
// symmetric positive definite system (D - d S) lambda = D c, solved here by
// conjugate gradients with the diagonal preconditioner D (Hestenes and
// Stiefel, 1952).  The preconditioned residual z = D^-1 r equals the Jacobi
// residual c + d A^T lambda - lambda, so the stopping rule is the same as the
// sweeps'.  Rows without weight (s = 0) keep lambda = c.  Vectors are fp32,
// dot products fp64; alpha, beta and the stop decision stay on the device.
struct CgState {
    double acc0, acc1;       // block partial sums of the running kernel
    double rz, alpha, beta, z1;
    double tol;
    unsigned blocks;
    int iters, max_iters, converged;
};

__device__ __forceinline__ float row_weight(const float *rs, int32_t v) {
    const float r = rs[v];
    return r > 0.f ? 1.0f / r : 0.f;
}

// Accumulates (a0, a1) over the grid; the last block to finish returns true
// in thread 0 with the totals in *t0, *t1 and the accumulators cleared.
__device__ __forceinline__ bool grid_sum2(CgState *cg, double a0, double a1, double *t0, double *t1) {
    __shared__ double s0[32], s1[32];
    __shared__ int s_last;
    a0 = block_sum(a0, s0);
    a1 = block_sum(a1, s1);
    if (threadIdx.x == 0) {
        if (a0 != 0.0) atomicAdd(&cg->acc0, a0);
        if (a1 != 0.0) atomicAdd(&cg->acc1, a1);
        __threadfence();
        s_last = atomicAdd(&cg->blocks, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return false;
    __threadfence();
    *t0 = *(volatile double *)&cg->acc0;
    *t1 = *(volatile double *)&cg->acc1;
    cg->acc0 = 0.0;
    cg->acc1 = 0.0;
    cg->blocks = 0;
    return true;
}

// r = s (c - lambda) + d S lambda, z = r / s, p = z; rz = r.z, stop if |z|_1 < tol.
__global__ void cg_start(int32_t n, const float *c, float *lam, const float *slam, const float *rs, float d, float *r,
                         float *p, CgState *cg, IterState *st) {
    double rz = 0.0, z1 = 0.0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float sv = row_weight(rs, v);
        if (sv == 0.f) {
            lam[v] = c[v];
            r[v] = 0.f;
            p[v] = 0.f;
            continue;
        }
        const float rv = sv * (c[v] - lam[v]) + d * slam[v];
        const float zv = rv * rs[v];
        r[v] = rv;
        p[v] = zv;
        rz += (double)rv * zv;
        z1 += fabs((double)zv);
    }
    double trz, tz1;
    if (grid_sum2(cg, rz, z1, &trz, &tz1)) {
        cg->rz = trz;
        cg->z1 = tz1;
        if (tz1 < cg->tol || trz <= 0.0) {
            cg->converged = 1;
            st->done = 1;
        }
    }
}

// alpha = rz / (p . q), p . q from the sweep's residual slot; lambda += alpha
// p, r -= alpha q; beta = r.z / rz; stop on |z|_1 < tol or the cap.
__global__ void cg_update(int32_t n, const float *p, const float *sp, const float *rs, float d, float *lam, float *r,
                          CgState *cg, IterState *st, int slot) {
    if (*(volatile int *)&st->done) return;
    const double pq = *(volatile double *)&st->l1[slot];
    if (!(pq > 0.0)) {  // p = 0 (already exact) or a breakdown: stop
        if (blockIdx.x == 0 && threadIdx.x == 0) st->done = 1;
        return;
    }
    const float alpha = (float)(cg->rz / pq);
    double rz = 0.0, z1 = 0.0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float pv = p[v];
        const float q = row_weight(rs, v) * pv - d * sp[v];
        lam[v] += alpha * pv;
        const float rv = r[v] - alpha * q;
        r[v] = rv;
        const float zv = rv * rs[v];
        rz += (double)rv * zv;
        z1 += fabs((double)zv);
    }
    double trz, tz1;
    if (grid_sum2(cg, rz, z1, &trz, &tz1)) {
        cg->beta = cg->rz > 0.0 ? trz / cg->rz : 0.0;
        cg->rz = trz;
        cg->z1 = tz1;
        cg->iters++;
        if (tz1 < cg->tol) cg->converged = 1;
        if (cg->converged || cg->iters >= cg->max_iters) st->done = 1;
    }
}

// p = z + beta p.
__global__ void cg_direction(int32_t n, const float *r, const float *rs, float *p, const CgState *cg,
                             const IterState *st) {
    if (*(volatile const int *)&st->done) return;
    const float beta = (float)cg->beta;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        p[v] = r[v] * rs[v] + beta * p[v];
}

// Solves the adjoint into lam (which holds the start) with the row plan's
// sweep for S x.  `work` holds 3 vectors of n floats.
hc_status run_cg(hc_graph *g, const PrPlanDev &plan, bool weighted, const float *c, float *lam, float d, double tol,
                 int max_iters, float *work, float *partials, unsigned *hub_count, SolveResult *res) {
    const int64_t n = g->N;
    float *r = work, *pv = work + n, *sp = work + 2 * n;
    IterState *st = reinterpret_cast<IterState *>(g->ws_ctl.ptr);
    CgState *cg = reinterpret_cast<CgState *>(g->ws_ctl.as<char>() + (sizeof(IterState) + 255) / 256 * 256);
    const float *rs = weighted ? g->inv_wsum.as<float>() : g->inv_deg.as<float>();
    HC_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(IterState), g->stream));
    CgState h{};
    h.tol = tol;
    h.max_iters = max_iters;
    HC_CUDA_TRY(cudaMemcpyAsync(cg, &h, sizeof(h), cudaMemcpyHostToDevice, g->stream));
    // y = S x through the pull sweep (own-row weights, no stopping rule of
    // its own: it returns at once once st->done is set); in the iterations
    // its epilogue also sums p . q (kCG).
    SweepArgs a{};
    a.index = g->index.as<int64_t>();
    a.nbr = g->nbr.as<int32_t>();
    a.ew = weighted ? pr_weights(g) : nullptr;
    a.base_scalar = 0.f;
    a.d = 1.0f;
    a.rs = rs;
    a.omega = 1.0f;
    a.partials = partials;
    a.hub_count = hub_count;
    a.st = st;
    a.tol_l1 = 0.f;
    a.eps = 3.4e38f;
    a.max_iters = max_iters;
    a.n_active = g->n_active;
    SweepFn sweep = pick_sweep(weighted, false, false, false);
    SweepFn cg_sweep = weighted ? launch_sweep<true, false, false, false, true> : launch_sweep<false, false, false, false, true>;
    const int grid = g->sm_count * 4;
    HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    a.it = 0;
    a.gin = lam;
    a.xin = sp;
    a.xout = sp;
    a.gout = sp;
    HC_TRY(sweep(g, a, plan));
    { cg_start<<<grid, 256, 0, g->stream>>>((int32_t)n, c, lam, sp, rs, d, r, pv, cg, st); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    constexpr int kRound = 4;
    HC_TRY(g->pinned.ensure(64));
    volatile int *hdone = g->pinned.as<int>();
    int it = 0;
    for (bool done = false; !done && it < max_iters;) {
        for (int k = 0; k < kRound && it < max_iters; k++, it++) {
            a.it = it + 1;
            a.gin = pv;
            a.d = d;
            HC_TRY(cg_sweep(g, a, plan));
            const int slot = a.it % kMaxIterSlots;
            { cg_update<<<grid, 256, 0, g->stream>>>((int32_t)n, pv, sp, rs, d, lam, r, cg, st, slot); ::hc::count_launch(); }
            { cg_direction<<<grid, 256, 0, g->stream>>>((int32_t)n, r, rs, pv, cg, st); ::hc::count_launch(); }
            HC_CUDA_TRY(cudaGetLastError());
        }
        HC_CUDA_TRY(cudaMemcpyAsync((void *)hdone, &st->done, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        done = *hdone != 0;
    }
    HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    HC_CUDA_TRY(cudaMemcpy(&h, cg, sizeof(h), cudaMemcpyDeviceToHost));
    res->iters = h.iters;
    res->done = h.converged;
    res->l1 = h.z1;
    res->changed = 0;
    HC_CUDA_TRY(cudaEventElapsedTime(&res->ms, g->ev_start, g->ev_stop));
    return HC_OK;
}

void fill_opts(const hc_pr_opts *opts, hc_pr_opts *o) {
    hc_pr_opts d{};
    if (opts) d = *opts;
    if (d.damping <= 0.f) d.damping = 0.85f;
    if (d.max_iters <= 0) d.max_iters = 50;
    if (d.tol_l1 < 0.f) d.tol_l1 = 0.f;
    if (d.eps_vertex < 0.f) d.eps_vertex = 0.f;
    if (d.tol_l1 == 0.f && d.eps_vertex == 0.f) d.tol_l1 = 1e-4f;
    *o = d;
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_pr_forward(hc_graph *g, const float *teleport, int32_t ncols, float *scores_out,
                                   const hc_pr_opts *opts, hc_pr_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    ReclaimScope reclaim_scope(g, kKeepPrWeighted);
    if (ncols < 1 || !scores_out) return fail(HC_ERR_INVALID_ARG, "hc_pr_forward: bad ncols / output");
    if (ncols > 1 && !teleport) return fail(HC_ERR_INVALID_ARG, "hc_pr_forward: ncols > 1 needs a teleport matrix");
    hc_pr_opts o;
    fill_opts(opts, &o);
    if (o.max_iters > kMaxIterSlots - 1) o.max_iters = kMaxIterSlots - 1;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const bool weighted = o.weighted != 0;
    HC_TRY(ensure_pr_derived(g, weighted));
    HC_TRY(ensure_plan(g));
    int partial_slots = 0;
    PrPlanDev plan = plan_view(g, &partial_slots);
    const int64_t n = g->N;
    HC_TRY(g->ws_ctl.ensure(sizeof(IterState) + 4096));

    if (ncols > 1) {
        // Dense multi-column form.
        const int K = ncols;
        const size_t nk = (size_t)n * K;
        const size_t bytes = 5 * nk * sizeof(float) + (size_t)(partial_slots + 1) * K * sizeof(float) +
                             (size_t)(plan.n_hub + 1) * 4 + (size_t)K * 8 + 4096;
        HC_TRY(g->ws_pr.ensure(bytes));
        char *p = g->ws_pr.as<char>();
        auto take = [&](size_t b) {
            char *r = p;
            p += (b + 255) / 256 * 256;
            return r;
        };
        float *basev = (float *)take(nk * 4);
        float *x[2] = {(float *)take(nk * 4), (float *)take(nk * 4)};
        float *gv[2] = {(float *)take(nk * 4), (float *)take(nk * 4)};
        float *partials = (float *)take((size_t)(partial_slots + 1) * K * 4);
        unsigned *hub_count = (unsigned *)take((size_t)(plan.n_hub + 1) * 4);
        double *col_l1 = (double *)take((size_t)K * 8);
        HC_TRY(copy_in(basev, teleport, nk * 4, g->stream));
        { scale_vec<<<g->sm_count * 8, 256, 0, g->stream>>>(basev, 1.0f - o.damping, basev, nk); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaMemsetAsync(hub_count, 0, (size_t)(plan.n_hub + 1) * 4, g->stream));
        const float *ps = weighted ? nullptr : g->inv_deg.as<float>();
        { spmm_init<<<g->sm_count * 8, 256, 0, g->stream>>>(g->N, K, basev, nullptr, nullptr, nullptr, o.damping, ps,
                                                          x[0], gv[0], x[1], gv[1], g->n_active); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        SpmmArgs a{};
        a.index = g->index.as<int64_t>();
        a.nbr = g->nbr.as<int32_t>();
        a.ew = weighted ? g->wtn.as<float>() : nullptr;
        a.basev = basev;
        a.d = o.damping;
        a.ps = ps;
        a.partials = partials;
        a.hub_count = hub_count;
        a.col_l1 = col_l1;
        a.K = K;
        a.n_active = g->n_active;
        HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
        int it = 0;
        std::vector<double> hl1(K);
        bool conv = false;
        for (; it < o.max_iters && !conv; it++) {
            a.gin = weighted ? x[it & 1] : gv[it & 1];
            a.xin = x[it & 1];
            a.xout = x[(it + 1) & 1];
            a.gout = weighted ? a.xout : gv[(it + 1) & 1];
            HC_CUDA_TRY(cudaMemsetAsync(col_l1, 0, (size_t)K * 8, g->stream));
            const int cols = (K + 31) / 32;
            const int grid = g->sm_count * 8;
            if (cols <= 1) { spmm_sweep<1><<<grid, kPrThreads, 0, g->stream>>>(a, plan, nullptr); ::hc::count_launch(); }
            else if (cols <= 2) { spmm_sweep<2><<<grid, kPrThreads, 0, g->stream>>>(a, plan, nullptr); ::hc::count_launch(); }
            else if (cols <= 4) { spmm_sweep<4><<<grid, kPrThreads, 0, g->stream>>>(a, plan, nullptr); ::hc::count_launch(); }
            else if (cols <= 8) { spmm_sweep<8><<<grid, kPrThreads, 0, g->stream>>>(a, plan, nullptr); ::hc::count_launch(); }
            else return fail(HC_ERR_UNSUPPORTED, "hc_pr_forward: at most 256 columns per call");
            HC_CUDA_TRY(cudaGetLastError());
            HC_CUDA_TRY(cudaMemcpyAsync(hl1.data(), col_l1, (size_t)K * 8, cudaMemcpyDeviceToHost, g->stream));
            HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
            double mx = 0;
            for (double v : hl1) mx = std::max(mx, v);
            conv = o.tol_l1 > 0.f && mx < (double)o.tol_l1;
        }
        HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
        HC_TRY(copy_out(scores_out, x[it & 1], nk * 4, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        float ms = 0;
        HC_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
        if (stats) {
            stats->iterations = it;
            stats->converged = conv;
            double mx = 0;
            for (double v : hl1) mx = std::max(mx, v);
            stats->residual_l1 = (float)mx;
            stats->ms = ms;
            stats->bytes_model = (double)it * (8.0 * (n + 1) + 4.0 * g->M * (weighted ? 2 : 1) +
                                               12.0 * (double)n * K);
        }
        return HC_OK;
    }

    const size_t bytes = 5 * (size_t)n * 4 + (size_t)(partial_slots + 1) * 4 + (size_t)(plan.n_hub + 1) * 4 + 4096;
    HC_TRY(g->ws_pr.ensure(bytes));
    char *p = g->ws_pr.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    float *basev = (float *)take(n * 4);
    float *x[2] = {(float *)take(n * 4), (float *)take(n * 4)};
    float *gv[2] = {(float *)take(n * 4), (float *)take(n * 4)};
    float *partials = (float *)take((size_t)(partial_slots + 1) * 4);
    unsigned *hub_count = (unsigned *)take((size_t)(plan.n_hub + 1) * 4);
    HC_CUDA_TRY(cudaMemsetAsync(hub_count, 0, (size_t)(plan.n_hub + 1) * 4, g->stream));
    bool cheb = false;
    if (o.accel == 1) HC_TRY(ensure_pr_symmetry(g, weighted, &cheb));
    const bool basevec = teleport != nullptr;
    if (basevec) {
        HC_TRY(copy_in(basev, teleport, n * 4, g->stream));
        { scale_vec<<<g->sm_count * 8, 256, 0, g->stream>>>(basev, 1.0f - o.damping, basev, (size_t)g->N); ::hc::count_launch(); }
    }
    // Uniform teleport: base (1-d)/N as the reference computes it
    // (src/kernels/gpu/pr.cuh:152), start from 1/N (src/kernels/cpu/pr.cuh:39).
    // A teleport vector t starts from t itself (base / (1-d)), which has the
    // fixed point's mass, so the error has no part in the slowest mode.
    const float base_scalar = (1.0f - o.damping) / (float)g->N;
    const float *ps = weighted ? nullptr : g->inv_deg.as<float>();
    { pr_init<<<g->sm_count * 8, 256, 0, g->stream>>>(g->N, basevec ? basev : nullptr, base_scalar,
                                                    basevec ? 0.f : 1.0f / (float)g->N, basevec ? basev : nullptr,
                                                    basevec ? 1.0f / (1.0f - o.damping) : 1.0f, ps, x[0], weighted ? nullptr : gv[0], x[1],
                                                    weighted ? nullptr : gv[1], g->n_active); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    SweepArgs a{};
    a.index = g->index.as<int64_t>();
    a.nbr = g->nbr.as<int32_t>();
    a.ew = weighted ? g->wtn.as<float>() : nullptr;
    a.basev = basev;
    a.base_scalar = base_scalar;
    a.d = o.damping;
    a.rs = nullptr;
    a.ps = ps;
    a.partials = partials;
    a.hub_count = hub_count;
    a.st = reinterpret_cast<IterState *>(g->ws_ctl.ptr);
    a.tol_l1 = o.tol_l1;
    a.eps = o.eps_vertex > 0.f ? o.eps_vertex : 3.4e38f;
    a.max_iters = o.max_iters;
    a.n_active = g->n_active;
    SweepFn fn = pick_sweep(weighted, false, !weighted, basevec);
    if (!fn) return fail(HC_ERR_UNSUPPORTED, "hc_pr_forward: no sweep for this option set");
    if (o.eps_vertex <= 0.f) a.eps = 3.4e38f;
    SolveResult r;
    HC_TRY(run_solve(g, a, plan, fn, x, gv, !weighted, &r, cheb ? o.damping : 0.f));
    HC_TRY(copy_out(scores_out, x[r.iters & 1], n * 4, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (stats) {
        stats->iterations = r.iters;
        stats->converged = r.done == 1;
        stats->residual_l1 = (float)r.l1;
        stats->changed = r.changed;
        stats->ms = r.ms;
        stats->bytes_model = (double)r.iters * (8.0 * (n + 1) + 4.0 * g->M * (weighted ? 2 : 1) + 12.0 * n);
    }
    return HC_OK;
}

extern "C" hc_status hc_pr_backward(hc_graph *g, const float *scores, const float *dL_dscores, float *dL_dteleport,
                                    float *dL_dweights, const hc_pr_opts *opts, hc_pr_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    ReclaimScope reclaim_scope(g, kKeepPrWeighted);
    if (!scores || !dL_dscores) return fail(HC_ERR_INVALID_ARG, "hc_pr_backward: scores and dL/dscores required");
    hc_pr_opts o;
    fill_opts(opts, &o);
    if (o.max_iters > kMaxIterSlots - 1) o.max_iters = kMaxIterSlots - 1;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const bool weighted = o.weighted != 0;
    HC_TRY(ensure_pr_derived(g, weighted));
    HC_TRY(ensure_plan(g));
    int partial_slots = 0;
    PrPlanDev plan = plan_view(g, &partial_slots);
    const int64_t n = g->N;
    HC_TRY(g->ws_ctl.ensure(sizeof(IterState) + sizeof(CgState) + 4096));
    // cvec, lam[2], xs, spare and the three vectors of the CG solve.
    const size_t bytes = 8 * (size_t)n * 4 + (size_t)(partial_slots + 1) * 4 + (size_t)(plan.n_hub + 1) * 4 + 8192;
    HC_TRY(g->ws_pr.ensure(bytes));
    char *p = g->ws_pr.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    float *cvec = (float *)take(n * 4);
    float *lam[2] = {(float *)take(n * 4), (float *)take(n * 4)};
    float *xs = (float *)take(n * 4);
    float *spare = (float *)take(n * 4);
    float *cg_work = (float *)take(3 * n * 4);  // r, p and S p of the conjugate-gradient solve
    float *partials = (float *)take((size_t)(partial_slots + 1) * 4);
    unsigned *hub_count = (unsigned *)take((size_t)(plan.n_hub + 1) * 4);
    HC_CUDA_TRY(cudaMemsetAsync(hub_count, 0, (size_t)(plan.n_hub + 1) * 4, g->stream));
    HC_TRY(copy_in(cvec, dL_dscores, n * 4, g->stream));
    HC_TRY(copy_in(xs, scores, n * 4, g->stream));
    // lambda_0 = c / (1-d); isolated vertices keep lambda = c.  With
    // symmetric weights the walk's stationary vector is the weighted degree
    // s, and the fixed point has s.lambda = s.c / (1-d) on every connected
    // component: this start already carries that, so the mode that decays
    // only at rate d (eigenvalue 1 of the walk) is absent from the start.
    // Any start converges to the same fixed point; this one converges fastest.
    { pr_init<<<g->sm_count * 8, 256, 0, g->stream>>>(g->N, cvec, 0.f, 0.f, cvec, 1.0f / (1.0f - o.damping), nullptr,
                                                    lam[0], nullptr, lam[1], nullptr, g->n_active); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    SweepArgs a{};
    a.index = g->index.as<int64_t>();
    a.nbr = g->nbr.as<int32_t>();
    a.ew = weighted ? pr_weights(g) : nullptr;
    a.basev = cvec;
    a.d = o.damping;
    a.rs = weighted ? g->inv_wsum.as<float>() : g->inv_deg.as<float>();
    a.ps = nullptr;
    a.partials = partials;
    a.hub_count = hub_count;
    a.st = reinterpret_cast<IterState *>(g->ws_ctl.ptr);
    // The adjoint's L1 rule is relative to sum |dL/dx| (lambda scales with it).
    {
        HC_TRY(g->pinned.ensure(64));
        double *hacc = g->pinned.as<double>();
        double *dacc = reinterpret_cast<double *>(spare);  // scratch until the solve ends
        HC_CUDA_TRY(cudaMemsetAsync(dacc, 0, sizeof(double), g->stream));
        { sum_abs<<<g->sm_count * 4, 256, 0, g->stream>>>(cvec, g->N, dacc); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaMemcpyAsync(hacc, dacc, sizeof(double), cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        a.tol_l1 = (float)(o.tol_l1 * *hacc);
    }
    a.eps = o.eps_vertex > 0.f ? o.eps_vertex : 3.4e38f;
    a.max_iters = o.max_iters;
    a.n_active = g->n_active;
    SweepFn fn = pick_sweep(weighted, true, false, true);
    // lambda = c + d A^T lambda.  For a reversible walk (symmetric weights)
    // A^T = D^-1 S is similar to a symmetric matrix with spectrum in [-1, 1]:
    // conjugate gradients on (D - d S) lambda = D c (accel 0 / 1), or Chebyshev
    // weights on the Jacobi sweeps, whose operator's spectrum lies in [-d, d]
    // (accel 2).  Otherwise, and with accel -1, plain Jacobi sweeps.
    bool sym = false;
    if (o.accel >= 0) HC_TRY(ensure_pr_symmetry(g, weighted, &sym));
    SolveResult r;
    float *lfin;
    if (sym && o.accel != 2) {
        HC_CUDA_TRY(cudaMemsetAsync(cg_work + 2 * n, 0, n * 4, g->stream));  // S p rows without edges stay 0
        HC_TRY(run_cg(g, plan, weighted, cvec, lam[0], o.damping, (double)a.tol_l1, o.max_iters, cg_work, partials,
                      hub_count, &r));
        lfin = lam[0];
    } else {
        float *gdummy[2] = {spare, spare};
        HC_TRY(run_solve(g, a, plan, fn, lam, gdummy, false, &r, sym ? o.damping : 0.f));
        lfin = lam[r.iters & 1];
    }
    HC_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    if (dL_dteleport) {
        const bool dev = is_device_pointer(dL_dteleport);
        float *dst = dev ? dL_dteleport : spare;
        { scale_vec<<<g->sm_count * 8, 256, 0, g->stream>>>(lfin, 1.0f - o.damping, dst, (size_t)g->N); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        if (!dev) HC_TRY(copy_out(dL_dteleport, spare, n * 4, g->stream));
    }
    if (dL_dweights) {
        const bool dev = is_device_pointer(dL_dweights);
        float *dst = dL_dweights;
        if (!dev) {
            HC_TRY(g->ws_out0.ensure(sizeof(float) * (size_t)std::max<int64_t>(g->M, 1)));
            dst = g->ws_out0.as<float>();
        }
        const float *rsv = weighted ? g->inv_wsum.as<float>() : g->inv_deg.as<float>();
        { pr_edge_grad<<<g->sm_count * 8, kPrThreads, 0, g->stream>>>(plan, a.index, a.nbr, rsv, xs, lfin, cvec,
                                                                      o.damping, g->n_active, dst); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        if (!dev) HC_TRY(copy_out(dL_dweights, dst, sizeof(float) * (size_t)g->M, g->stream));
    }
    HC_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    float ms2 = 0;
    HC_CUDA_TRY(cudaEventElapsedTime(&ms2, g->ev_start, g->ev_stop));
    if (stats) {
        stats->iterations = r.iters;
        stats->converged = r.done == 1;
        stats->residual_l1 = (float)r.l1;
        stats->changed = r.changed;
        stats->ms = r.ms + ms2;
        stats->bytes_model = (double)r.iters * (8.0 * (n + 1) + 4.0 * g->M * (weighted ? 2 : 1) + 12.0 * n) +
                             (dL_dweights ? (8.0 * (n + 1) + 4.0 * g->M * (weighted ? 3 : 2) + 8.0 * n) : 0.0);
    }
    return HC_OK;
}

extern "C" hc_status hc_ppr_batched(hc_graph *g, const int32_t *seed_offsets, const int32_t *seeds, int32_t ncols,
                                    float *scores_out, const hc_pr_opts *opts, hc_pr_stats *stats) {
    clear_error();
    HC_TRY(activate(g));
    ReclaimScope reclaim_scope(g, kKeepPrWeighted | kKeepBatch);
    if (ncols < 1 || ncols > 256 || !seed_offsets || !seeds || !scores_out)
        return fail(HC_ERR_INVALID_ARG, "hc_ppr_batched: bad arguments (1 <= ncols <= 256)");
    hc_pr_opts o;
    fill_opts(opts, &o);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    const bool weighted = o.weighted != 0;
    HC_TRY(ensure_pr_derived(g, weighted));
    HC_TRY(ensure_plan(g));
    int partial_slots = 0;
    PrPlanDev plan = plan_view(g, &partial_slots);
    std::vector<int32_t> off(ncols + 1);
    HC_CUDA_TRY(cudaMemcpy(off.data(), seed_offsets, sizeof(int32_t) * (ncols + 1), cudaMemcpyDefault));
    if (off[0] != 0) return fail(HC_ERR_INVALID_ARG, "hc_ppr_batched: seed_offsets[0] must be 0");
    for (int c = 0; c < ncols; c++)
        if (off[c + 1] <= off[c]) return fail(HC_ERR_INVALID_ARG, "hc_ppr_batched: column %d has no seed", c);
    const int32_t nseeds = off[ncols];
    std::vector<int32_t> sd(nseeds);
    HC_CUDA_TRY(cudaMemcpy(sd.data(), seeds, sizeof(int32_t) * nseeds, cudaMemcpyDefault));
    for (int32_t s : sd)
        if (s < 0 || s >= g->N) return fail(HC_ERR_INVALID_ARG, "hc_ppr_batched: seed %d out of range", s);
    const int K = ncols;
    const int64_t n = g->N;
    const size_t nk = (size_t)n * K;
    const size_t bytes = 4 * nk * sizeof(float) + (size_t)(partial_slots + 1) * K * 4 + (size_t)(plan.n_hub + 1) * 4 +
                         (size_t)K * 8 + (size_t)n + (size_t)(nseeds + ncols + 1) * 4 + 5 * (size_t)n * 4 + 16384;
    HC_TRY(g->ws_pr.ensure(bytes));
    char *p = g->ws_pr.as<char>();
    auto take = [&](size_t b) {
        char *r = p;
        p += (b + 255) / 256 * 256;
        return r;
    };
    float *x[2] = {(float *)take(nk * 4), (float *)take(nk * 4)};
    float *gv[2] = {(float *)take(nk * 4), (float *)take(nk * 4)};
    float *partials = (float *)take((size_t)(partial_slots + 1) * K * 4);
    unsigned *hub_count = (unsigned *)take((size_t)(plan.n_hub + 1) * 4);
    double *col_l1 = (double *)take((size_t)K * 8);
    uint8_t *is_seed = (uint8_t *)take((size_t)n);
    int32_t *d_off = (int32_t *)take((size_t)(ncols + 1) * 4);
    int32_t *d_seeds = (int32_t *)take((size_t)nseeds * 4);
    float *col_x[2] = {(float *)take((size_t)n * 4), (float *)take((size_t)n * 4)};
    float *col_g[2] = {(float *)take((size_t)n * 4), (float *)take((size_t)n * 4)};
    float *col_base = (float *)take((size_t)n * 4);
    HC_CUDA_TRY(cudaMemcpyAsync(d_off, off.data(), (ncols + 1) * 4, cudaMemcpyHostToDevice, g->stream));
    HC_CUDA_TRY(cudaMemcpyAsync(d_seeds, sd.data(), (size_t)nseeds * 4, cudaMemcpyHostToDevice, g->stream));
    HC_CUDA_TRY(cudaMemsetAsync(is_seed, 0, (size_t)n, g->stream));
    HC_CUDA_TRY(cudaMemsetAsync(hub_count, 0, (size_t)(plan.n_hub + 1) * 4, g->stream));
    { mark_seeds<<<64, 256, 0, g->stream>>>(d_seeds, nseeds, is_seed); ::hc::count_launch(); }
    const float *ps = weighted ? nullptr : g->inv_deg.as<float>();
    { spmm_init<<<g->sm_count * 8, 256, 0, g->stream>>>(g->N, K, nullptr, d_off, d_seeds, is_seed, o.damping, ps,
                                                      x[0], gv[0], x[1], gv[1], g->n_active); ::hc::count_launch(); }
    HC_CUDA_TRY(cudaGetLastError());
    SpmmArgs a{};
    a.index = g->index.as<int64_t>();
    a.nbr = g->nbr.as<int32_t>();
    a.ew = weighted ? g->wtn.as<float>() : nullptr;
    a.basev = nullptr;
    a.seed_off = d_off;
    a.seed_idx = d_seeds;
    a.d = o.damping;
    a.ps = ps;
    a.partials = partials;
    a.hub_count = hub_count;
    a.col_l1 = col_l1;
    a.K = K;
    a.n_active = g->n_active;
    // Columns converge at their own pace (personalised teleports differ):
    // a column whose L1 change falls below tol is final.  Whenever the live
    // columns fit fewer 32-column chunks, one pass writes the final ones to
    // the output and packs the live ones tighter, so later sweeps gather only
    // live columns.
    const bool dev_out = is_device_pointer(scores_out);
    float *out = scores_out;
    if (!dev_out) {
        HC_TRY(g->ws_out0.ensure(nk * 4));
        out = g->ws_out0.as<float>();
    }
    HC_TRY(g->ws_src.ensure((size_t)2 * K * 4));
    int32_t *d_map = g->ws_src.as<int32_t>();
    int32_t *d_newpos = d_map + K;
    std::vector<int32_t> hmap(K), hpos(K);
    for (int c = 0; c < K; c++) hmap[c] = c;
    HC_CUDA_TRY(cudaMemcpyAsync(d_map, hmap.data(), (size_t)K * 4, cudaMemcpyHostToDevice, g->stream));
    a.col_map = d_map;
    auto repack = [&](int cur, int kw, int nkw) -> hc_status {
        HC_CUDA_TRY(cudaMemcpyAsync(d_newpos, hpos.data(), (size_t)kw * 4, cudaMemcpyHostToDevice, g->stream));
        {
            spmm_repack<<<g->sm_count * 8, 256, 0, g->stream>>>(g->N, kw, x[cur], d_newpos, d_map, K, out, nkw,
                                                                x[cur ^ 1], weighted ? nullptr : gv[cur ^ 1], ps);
            ::hc::count_launch();
        }
        HC_CUDA_TRY(cudaGetLastError());
        // Rows without edges (past n_active) are never written by a sweep:
        // give the buffer the next sweep writes their values in the new layout.
        if (nkw > 0 && g->n_active < g->N)
            HC_CUDA_TRY(cudaMemcpyAsync(x[cur] + (size_t)g->n_active * nkw, x[cur ^ 1] + (size_t)g->n_active * nkw,
                                        (size_t)(g->N - g->n_active) * nkw * 4, cudaMemcpyDeviceToDevice, g->stream));
        return HC_OK;
    };
    // The single-column solver's run_solve records g's events: this call
    // times itself with its own pair.
    cudaEvent_t ev0, ev1;
    HC_CUDA_TRY(cudaEventCreate(&ev0));
    HC_CUDA_TRY(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } ev_guard{ev0, ev1};
    HC_CUDA_TRY(cudaEventRecord(ev0, g->stream));
    int it = 0, cur = 0, kw = K;
    std::vector<double> hl1(K);
    double bytes_model = 0, mx = 0;
    bool conv = false;
    // A few slow columns (a seed set in a small bipartite component converges
    // at rate d) finish on the single-column sweeps, which gather 4 bytes per
    // edge instead of a 32-column row segment.
    constexpr int kSingleCols = 4;
    for (; it < o.max_iters && kw > (K > kSingleCols ? kSingleCols : 0); it++) {
        a.K = kw;
        a.gin = weighted ? x[cur] : gv[cur];
        a.xin = x[cur];
        a.xout = x[cur ^ 1];
        a.gout = weighted ? a.xout : gv[cur ^ 1];
        HC_CUDA_TRY(cudaMemsetAsync(col_l1, 0, (size_t)kw * 8, g->stream));
        const int cols = (kw + 31) / 32;
        const int grid = g->sm_count * 8;
        if (cols <= 1) { spmm_sweep<1><<<grid, kPrThreads, 0, g->stream>>>(a, plan, is_seed); ::hc::count_launch(); }
        else if (cols <= 2) { spmm_sweep<2><<<grid, kPrThreads, 0, g->stream>>>(a, plan, is_seed); ::hc::count_launch(); }
        else if (cols <= 4) { spmm_sweep<4><<<grid, kPrThreads, 0, g->stream>>>(a, plan, is_seed); ::hc::count_launch(); }
        else { spmm_sweep<8><<<grid, kPrThreads, 0, g->stream>>>(a, plan, is_seed); ::hc::count_launch(); }
        HC_CUDA_TRY(cudaGetLastError());
        bytes_model += 8.0 * (n + 1) + 4.0 * g->M * (weighted ? 2 : 1) + 12.0 * (double)n * kw;
        cur ^= 1;
        HC_CUDA_TRY(cudaMemcpyAsync(hl1.data(), col_l1, (size_t)kw * 8, cudaMemcpyDeviceToHost, g->stream));
        HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
        int live = 0;
        mx = 0;
        for (int c = 0; c < kw; c++) {
            mx = std::max(mx, hl1[c]);
            const bool done = o.tol_l1 > 0.f && hl1[c] < (double)o.tol_l1;
            hpos[c] = done ? -1 : live++;
        }
        if (live == 0) {
            conv = true;
            HC_TRY(repack(cur, kw, 0));  // every column is final
            kw = 0;
        } else if ((live + 31) / 32 < (kw + 31) / 32 || (live <= kSingleCols && kw > kSingleCols)) {
            HC_TRY(repack(cur, kw, live));
            std::vector<int32_t> nmap(live);
            for (int c = 0; c < kw; c++)
                if (hpos[c] >= 0) nmap[hpos[c]] = hmap[c];
            HC_CUDA_TRY(cudaStreamSynchronize(g->stream));  // d_map is read by the repack
            hmap = nmap;
            HC_CUDA_TRY(cudaMemcpyAsync(d_map, hmap.data(), (size_t)live * 4, cudaMemcpyHostToDevice, g->stream));
            cur ^= 1;
            kw = live;
        }
    }
    int tail_iters = 0;
    if (kw > 0 && it < o.max_iters) {
        // Each remaining column continues from its packed values on the
        // single-column sweeps (teleport vector, same stopping rule).
        SweepArgs sa{};
        sa.index = g->index.as<int64_t>();
        sa.nbr = g->nbr.as<int32_t>();
        sa.ew = weighted ? g->wtn.as<float>() : nullptr;
        sa.basev = col_base;
        sa.d = o.damping;
        sa.ps = ps;
        sa.partials = partials;
        sa.hub_count = hub_count;
        sa.st = reinterpret_cast<IterState *>(g->ws_ctl.ptr);
        sa.tol_l1 = o.tol_l1;
        sa.eps = 3.4e38f;
        sa.max_iters = o.max_iters - it;
        sa.n_active = g->n_active;
        SweepFn fn = pick_sweep(weighted, false, !weighted, true);
        HC_TRY(g->ws_ctl.ensure(sizeof(IterState) + 4096));
        sa.st = reinterpret_cast<IterState *>(g->ws_ctl.ptr);
        bool all_conv = true;
        for (int c = 0; c < kw; c++) {
            const int oc = hmap[c];
            HC_CUDA_TRY(cudaMemsetAsync(col_base, 0, (size_t)n * 4, g->stream));
            { spmm_column_base<<<4, 256, 0, g->stream>>>(d_seeds, off[oc], off[oc + 1], 1.0f - o.damping, col_base); ::hc::count_launch(); }
            {
                spmm_take_column<<<g->sm_count * 4, 256, 0, g->stream>>>(g->N, kw, c, x[cur], ps, col_x[0], col_x[1],
                                                                         weighted ? nullptr : col_g[0],
                                                                         weighted ? nullptr : col_g[1]);
                ::hc::count_launch();
            }
            HC_CUDA_TRY(cudaGetLastError());
            SolveResult r;
            HC_TRY(run_solve(g, sa, plan, fn, col_x, col_g, !weighted, &r));
            { spmm_put_column<<<g->sm_count * 4, 256, 0, g->stream>>>(g->N, col_x[r.iters & 1], K, oc, out); ::hc::count_launch(); }
            HC_CUDA_TRY(cudaGetLastError());
            tail_iters = std::max(tail_iters, r.iters);
            all_conv = all_conv && r.done == 1;
            mx = std::max(mx, r.l1);
            bytes_model += (double)r.iters * (8.0 * (n + 1) + 4.0 * g->M * (weighted ? 2 : 1) + 12.0 * (double)n);
        }
        conv = all_conv;
        kw = 0;
    }
    if (kw > 0) {  // iteration cap: the live columns as they stand
        for (int c = 0; c < kw; c++) hpos[c] = -1;
        HC_TRY(repack(cur, kw, 0));
    }
    HC_CUDA_TRY(cudaEventRecord(ev1, g->stream));
    if (!dev_out) HC_TRY(copy_out(scores_out, out, nk * 4, g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    float ms = 0;
    HC_CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
    if (stats) {
        stats->iterations = it + tail_iters;
        stats->converged = conv;
        stats->residual_l1 = (float)mx;
        stats->ms = ms;
        stats->bytes_model = bytes_model;
    }
    return HC_OK;
}
