/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY.  A CPU restatement of the reference's
 * algorithms for the epoch-kernel path, used by tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg as the checker.  Nothing in the product
 * (hetero-compute_b200/) links, loads or calls this file.
 *
 * Each function names the reference code it restates (paths inside
 * chrisliu/hetero-compute).  Pinned against the reference's own CPU code,
 * compiled unchanged from its sources by oracle/Makefile into oracle/_ref/,
 * through the golden fixtures in tests/golden/ (tests/test_oracle.py).
 *
 * Single-threaded on purpose: `cores` = 1 when timed as the port baseline.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define INVALID (-1)

/* Serial breadth-first depths: tests/bfs/bfs_verify.cu:211-233
 * (compute_proper_depth).  depth[v] = -1 when unreached. */
int or_bfs_depth(const int64_t *index, const int32_t *nbr, int32_t n, int32_t src, int32_t *depth) {
    int32_t *queue = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    if (!queue) return -1;
    for (int32_t i = 0; i < n; i++) depth[i] = INVALID;
    depth[src] = 0;
    int64_t head = 0, tail = 0;
    queue[tail++] = src;
    while (head < tail) {
        int32_t u = queue[head++];
        for (int64_t e = index[u]; e < index[u + 1]; e++) {
            int32_t v = nbr[e];
            if (depth[v] == INVALID) {
                depth[v] = depth[u] + 1;
                queue[tail++] = v;
            }
        }
    }
    free(queue);
    return 0;
}

/* Parent-array validation: tests/bfs/bfs_verify.cu:133-197 (verify_parents).
 * counts[0..3] = bad source, bad unexplored, explored too shallow, explored
 * too deep.  Additionally (not in the reference) requires parent[v] to be an
 * actual neighbour of v, which the depth rule alone does not check.
 * Returns the total number of errors. */
int64_t or_verify_bfs_parents(const int64_t *index, const int32_t *nbr, const int32_t *depth,
                              const int32_t *parents, int32_t n, int32_t src, int64_t *counts) {
    int64_t c[5] = {0, 0, 0, 0, 0};
    for (int32_t u = 0; u < n; u++) {
        int32_t p = parents[u];
        if (p == INVALID) {
            if (depth[u] != INVALID) c[1]++;
        } else if (u == src) {
            if (p != src) c[0]++;
        } else if (p < 0 || p >= n || depth[p] == INVALID || depth[u] != depth[p] + 1) {
            if (p >= 0 && p < n && depth[p] != INVALID && depth[u] < depth[p] + 1) c[2]++;
            else c[3]++;
        } else {
            int found = 0;
            for (int64_t e = index[u]; e < index[u + 1] && !found; e++) found = nbr[e] == p;
            if (!found) c[4]++;
        }
    }
    if (counts) memcpy(counts, c, sizeof(c));
    return c[0] + c[1] + c[2] + c[3] + c[4];
}

/* ----------------------------------------------------------------- SSSP */

typedef struct { int64_t d; int32_t v; } HeapItem;

static void heap_push(HeapItem *h, int64_t *sz, HeapItem x) {
    int64_t i = (*sz)++;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (h[p].d <= x.d) break;
        h[i] = h[p];
        i = p;
    }
    h[i] = x;
}

static HeapItem heap_pop(HeapItem *h, int64_t *sz) {
    HeapItem top = h[0], x = h[--(*sz)];
    int64_t i = 0;
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        int64_t md = x.d;
        if (l < *sz && h[l].d < md) { m = l; md = h[l].d; }
        if (r < *sz && h[r].d < md) { m = r; }
        if (m == i) break;
        h[i] = h[m];
        i = m;
    }
    h[i] = x;
    return top;
}

/* Dijkstra with a binary heap and lazy deletion:
 * src/kernels/cpu/sssp.cuh:74-109 (sssp_dijkstras_cpu_serial), integer
 * weights.  dist[v] = INT32_MAX when unreachable. */
int or_sssp_dijkstra(const int64_t *index, const int32_t *nbr, const int32_t *w, int32_t n, int32_t src,
                     int32_t *dist) {
    int64_t m = index[n];
    HeapItem *heap = (HeapItem *)malloc(sizeof(HeapItem) * (size_t)(m + 2));
    int64_t *d = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (!heap || !d) { free(heap); free(d); return -1; }
    for (int32_t i = 0; i < n; i++) d[i] = INT64_MAX;
    int64_t sz = 0;
    d[src] = 0;
    HeapItem s0 = {0, src};
    heap_push(heap, &sz, s0);
    while (sz > 0) {
        HeapItem it = heap_pop(heap, &sz);
        if (it.d != d[it.v]) continue;
        for (int64_t e = index[it.v]; e < index[it.v + 1]; e++) {
            int64_t nd = it.d + w[e];
            int32_t v = nbr[e];
            if (nd < d[v]) {
                d[v] = nd;
                HeapItem x = {nd, v};
                heap_push(heap, &sz, x);
            }
        }
    }
    for (int32_t i = 0; i < n; i++) dist[i] = d[i] == INT64_MAX ? INT32_MAX : (int32_t)d[i];
    free(heap);
    free(d);
    return 0;
}

/* Shortest-path-tree check: every reached v != src has a parent p with an
 * edge p -> v of weight w and dist[p] + w == dist[v]; unreached vertices have
 * parent -1; parent[src] == src.  Returns the number of violations. */
int64_t or_verify_sp_tree(const int64_t *index, const int32_t *nbr, const int32_t *w, const int32_t *dist,
                          const int32_t *parent, int32_t n, int32_t src) {
    int64_t bad = 0;
    for (int32_t v = 0; v < n; v++) {
        int32_t p = parent[v];
        if (v == src) { bad += p != src; continue; }
        if (dist[v] == INT32_MAX) { bad += p != INVALID; continue; }
        if (p < 0 || p >= n || dist[p] == INT32_MAX) { bad++; continue; }
        int ok = 0;
        for (int64_t e = index[p]; e < index[p + 1] && !ok; e++)
            ok = nbr[e] == v && (int64_t)dist[p] + w[e] == (int64_t)dist[v];
        bad += !ok;
    }
    return bad;
}

/* ------------------------------------------------------------- PageRank */

/* pr_pull_cpu with epoch_pr_pull_cpu_one_to_one on one thread:
 * src/kernels/cpu/pr.cuh:33-65 and :157-187.  Scores start at 1/N as the
 * CPU reference does (it ignores init_scores), or at init_scores when given
 * (the caller's init_score of pr_pull_gpu, src/kernels/gpu/pr.cuh:42-46,
 * 77-80); each sweep updates in place in vertex
 * order: new = (1 - d)/N + d * sum_u score[u]/deg(u) in float, written only
 * when |new - old| > eps; stops after a sweep with no write, or after
 * max_iters sweeps (the CPU reference has no cap).  Returns the sweeps run. */
int32_t or_pr_pull(const int64_t *index, const int32_t *nbr, int32_t n, float damping, float eps,
                   int32_t max_iters, const float *init_scores, float *score) {
    const float init = 1.0f / (float)n;
    const float base = (1.0f - damping) / (float)n;
    for (int32_t i = 0; i < n; i++) score[i] = init_scores ? init_scores[i] : init;
    int32_t it = 0;
    for (;;) {
        int64_t updated = 0;
        for (int32_t v = 0; v < n; v++) {
            float total = 0.0f;
            for (int64_t e = index[v]; e < index[v + 1]; e++) {
                int32_t u = nbr[e];
                total += score[u] / (float)(index[u + 1] - index[u]);
            }
            float ns = base + damping * total;
            if (fabsf(ns - score[v]) > eps) {
                score[v] = ns;
                updated++;
            }
        }
        it++;
        if (updated == 0 || (max_iters > 0 && it >= max_iters)) break;
    }
    return it;
}

/* FP64 Jacobi fixed point x = (1-d) t + d A x, A[v,u] = W_uv where W_uv =
 * w_uv / sum_k w_uk (w = NULL: 1/deg(u)); t = NULL means uniform 1/N.  Runs
 * until the L1 change drops below tol or max_iters.  Returns iterations. */
int32_t or_pr_jacobi_f64(const int64_t *index, const int32_t *nbr, const float *w, int32_t n,
                         const double *teleport, double damping, double tol, int32_t max_iters, double *x) {
    double *y = (double *)malloc(sizeof(double) * (size_t)n);
    double *inv = (double *)malloc(sizeof(double) * (size_t)n);
    if (!y || !inv) { free(y); free(inv); return -1; }
#pragma omp parallel for schedule(static)
    for (int32_t u = 0; u < n; u++) {
        double s = 0.0;
        for (int64_t e = index[u]; e < index[u + 1]; e++) s += w ? (double)w[e] : 1.0;
        inv[u] = s > 0.0 ? 1.0 / s : 0.0;
    }
    for (int32_t v = 0; v < n; v++) x[v] = teleport ? teleport[v] : 1.0 / n;
    int32_t it = 0;
    for (; it < max_iters; it++) {
        double l1 = 0.0;
        /* Each y[v] is one thread's sequential row sum, so x does not depend
         * on the thread count; only the L1 total's rounding does. */
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : l1)
        for (int32_t v = 0; v < n; v++) {
            double acc = 0.0;
            for (int64_t e = index[v]; e < index[v + 1]; e++) {
                int32_t u = nbr[e];
                double wuv = 1.0;
                if (w) {
                    /* weight of u -> v lives in row u */
                    wuv = 0.0;
                    for (int64_t f = index[u]; f < index[u + 1]; f++)
                        if (nbr[f] == v) { wuv = (double)w[f]; break; }
                }
                acc += wuv * inv[u] * x[u];
            }
            double t = teleport ? teleport[v] : 1.0 / n;
            y[v] = (1.0 - damping) * t + damping * acc;
            l1 += fabs(y[v] - x[v]);
        }
        memcpy(x, y, sizeof(double) * (size_t)n);
        if (l1 < tol) { it++; break; }
    }
    free(y);
    free(inv);
    return it;
}
