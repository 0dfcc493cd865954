/*
 * hc.h -- C ABI of the B200-native epoch-kernel engine (BFS, SSSP, PageRank).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, never
 * exits the process and reports failure through an hc_status code plus a
 * thread-local message (hc_last_error).  Array arguments may be host or device
 * pointers unless stated otherwise: the library inspects each pointer and
 * copies through HBM as needed.
 *
 * Reference interfaces replaced (paths inside chrisliu/hetero-compute):
 *   graph container / loader ........ src/graph.cuh:43-100, :207-239
 *   SourcePicker .................... src/graph.cuh:106-141
 *   epoch-kernel typedefs ........... src/kernels/kernel_types.cuh:29-63
 *   bfs_gpu driver .................. src/kernels/gpu/bfs.cuh:21-95
 *   sssp_pull_gpu driver ............ src/kernels/gpu/sssp.cuh:42-100
 *   pr_pull_gpu driver .............. src/kernels/gpu/pr.cuh:42-118
 *   CUDA_ERRCHK / CONDCHK (abort) ... src/cuda.cuh:14-21, src/util.h:16-22
 */
#ifndef HC_H
#define HC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Replaces the reference's print-and-exit error macros
 * (src/cuda.cuh:14-21, src/util.h:16-22). */
typedef enum hc_status {
    HC_OK = 0,
    HC_ERR_INVALID_ARG = 1,
    HC_ERR_OOM = 2,
    HC_ERR_CUDA = 3,
    HC_ERR_NOT_CONVERGED = 4, /* iteration / epoch cap reached */
    HC_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up */
    HC_ERR_NO_DEVICE = 6,
    HC_ERR_UNSUPPORTED = 7,
    HC_ERR_IO = 8
} hc_status;

/* Edge-weight storage.  The reference keeps weights interleaved with the
 * neighbour id as float (wnode_t, src/graph.cuh:37-41); here they are a
 * separate array (SoA) of int32 (SSSP) or fp32 (weighted PageRank). */
typedef enum hc_wtype { HC_W_NONE = 0, HC_W_I32 = 1, HC_W_F32 = 2 } hc_wtype;

/* Epoch-kernel granularity.  Reference registries: BFSGPU
 * (src/kernels/gpu/bfs.cuh:295-298), SSSPGPU (src/kernels/gpu/sssp.cuh:287-289),
 * PRGPU (src/kernels/gpu/pr.cuh:324-326): one_to_one = THREAD,
 * warp / warp_red = WARP, block_red = BLOCK.  AUTO lets the per-epoch
 * selector choose. */
typedef enum hc_variant {
    HC_VARIANT_AUTO = 0,
    HC_VARIANT_THREAD = 1,
    HC_VARIANT_WARP = 2,
    HC_VARIANT_BLOCK = 3
} hc_variant;

/* Host CSR graph: int64 offsets, int32 neighbours (GenericCSRGraph,
 * src/graph.cuh:43-86).  Arrays owned by the library when produced by
 * hc_gen_* / hc_csr_read and released with hc_csr_free. */
typedef struct hc_csr {
    int32_t num_nodes;
    int64_t num_edges;  /* directed edges = length of neighbors */
    int64_t *index;     /* num_nodes + 1 */
    int32_t *neighbors; /* num_edges */
    void *weights;      /* num_edges int32 or float, or NULL */
    hc_wtype wtype;
} hc_csr;

const char *hc_last_error(void);
const char *hc_status_string(hc_status s);
int32_t hc_abi_version(void);

/* ---------------------------------------------------------------- graphs */

/* Kronecker / R-MAT (A=.57, B=.19, C=.19), 2^scale vertices,
 * edge_factor * 2^scale generated pairs, random id permutation,
 * symmetrized, self-loops and duplicates removed (the lightest weight of a
 * duplicate set is kept), relabelled by descending degree, rows sorted.
 * Semantics of the reference's gapbs adapters: src/gapbs/generator.h:82-115,
 * src/gapbs/builder.h:141-186, :366-406.  Weights: HC_W_I32 uniform [1,255]
 * (src/gapbs/generator.h:133-147), HC_W_F32 uniform (0,1]. */
hc_status hc_gen_kronecker(int32_t scale, int32_t edge_factor, uint64_t seed,
                           hc_wtype wtype, hc_csr *out);
/* Erdos-Renyi: uniform endpoints (src/gapbs/generator.h:65-80), same build. */
hc_status hc_gen_uniform(int32_t scale, int32_t degree, uint64_t seed,
                         hc_wtype wtype, hc_csr *out);
/* rows x cols 4-neighbour grid, id = r * cols + c, symmetric weights. */
hc_status hc_gen_grid(int32_t rows, int32_t cols, uint64_t seed, hc_wtype wtype,
                      hc_csr *out);
void hc_csr_free(hc_csr *g);
/* .sg / .wsg binary format (src/graph.cuh:207-224):
 * [int32 N][int64 M][int64 index[N+1]][M x (int32 v) or M x (int32 v, float w)]. */
hc_status hc_csr_read(const char *path, int32_t weighted, hc_csr *out);
hc_status hc_csr_write(const char *path, const hc_csr *g);
/* SourcePicker (src/graph.cuh:106-141): mt19937 seeded 37525, uniform over
 * [0, N-1], rejecting degree-0 and self-loop-only vertices.  const_source >= 0
 * repeats that vertex.  Host arrays only. */
hc_status hc_pick_sources(const int64_t *index, const int32_t *neighbors,
                          int32_t num_nodes, int32_t count, int32_t const_source,
                          int32_t *out);

/* ---------------------------------------------------------- device graph */

typedef struct hc_graph hc_graph;

typedef struct hc_graph_info {
    int32_t num_nodes;
    int64_t num_edges;
    int32_t num_active;     /* vertices with degree > 0 (prefix when degree-sorted) */
    int32_t degree_sorted;  /* 1 if degrees are non-increasing in vertex id */
    int32_t max_degree;
    int32_t device;
    hc_wtype wtype;
    int64_t device_bytes;   /* HBM held by the handle */
} hc_graph_info;

/* Upload a CSR graph once (the reference re-uploads per driver call,
 * src/kernels/gpu/sssp.cuh:51-61).  Inputs may be host or device pointers. */
hc_status hc_graph_create(const int64_t *index, const int32_t *neighbors,
                          const void *weights, hc_wtype wtype, int32_t num_nodes,
                          int64_t num_edges, int32_t device, hc_graph **out);
hc_status hc_graph_destroy(hc_graph *g);

/* A .sg / .wsg file (layout as hc_csr_read; weighted 0 = .sg, 1 = .wsg with
 * fp32 weights, 2 = .wsg with weights converted to int32, which must be
 * non-negative integers) streamed into a device graph on `device`: chunks
 * go through two pinned staging buffers, file reads overlapping the copies,
 * so host memory stays at 64 MB whatever the graph's size.  Checked like
 * hc_graph_create; a short or inconsistent file returns HC_ERR_IO.  Replaces
 * load_graph_from_file (src/graph.cuh:207-239) plus the drivers' per-call
 * upload (src/kernels/gpu/sssp.cuh:51-61). */
hc_status hc_graph_load(const char *path, int32_t weighted, int32_t device, hc_graph **out);

/* Synthetic graphs built on the device: the same CSR as hc_gen_kronecker /
 * hc_gen_uniform (same scale, edge factor or pairs per vertex, seed and
 * weights) followed by hc_graph_create, without host memory or an upload.
 * Replaces the host-side build of the reference's gapbs adapters
 * (src/gapbs/generator.h:53-165, src/gapbs/builder.h:80-406). */
typedef enum hc_gen_kind { HC_GEN_KRONECKER = 0, HC_GEN_UNIFORM = 1 } hc_gen_kind;
hc_status hc_graph_generate(hc_gen_kind kind, int32_t scale, int32_t edge_factor, uint64_t seed,
                            hc_wtype wtype, int32_t device, hc_graph **out);
/* Copies the handle's CSR into caller buffers (host or device; any may be
 * NULL): index [N+1], neighbors [M], weights [M] (4-byte values). */
hc_status hc_graph_get_csr(hc_graph *g, int64_t *index, int32_t *neighbors, void *weights);
/* hc_pick_sources on a handle's graph (reads its offsets, and the neighbour of
 * each degree-1 candidate, from the device). */
hc_status hc_graph_pick_sources(hc_graph *g, int32_t count, int32_t *out);
/* Work of this handle goes to `stream` (a cudaStream_t); NULL restores the
 * handle's own stream. */
hc_status hc_graph_set_stream(hc_graph *g, void *stream);
hc_status hc_graph_get_info(const hc_graph *g, hc_graph_info *info);

/* ------------------------------------------------------------------- BFS */

typedef struct hc_bfs_opts {
    int32_t alpha;        /* top-down -> bottom-up when m_f > m_u / alpha (0: 15) */
    int32_t beta;         /* bottom-up -> top-down when n_f < N / beta (0: 18) */
    int32_t direction;    /* 0 auto (direction-optimising), 1 top-down only, 2 bottom-up only */
    hc_variant bu_variant;/* bottom-up granularity: THREAD (= AUTO) thread per vertex;
                             WARP warp per vertex; BLOCK warp per vertex for the
                             degree >= 32 prefix of a degree-sorted graph, thread after */
    int32_t collect_stats;/* count scanned vertices / edges (slower) */
} hc_bfs_opts;

typedef struct hc_bfs_stats {
    int32_t levels;
    int32_t td_levels;
    int32_t bu_levels;
    int32_t reached;
    int64_t vertices_scanned;
    int64_t edges_scanned;
    double bytes_model;   /* algorithmic bytes, summed over sources */
    double ms;            /* device time, summed over sources */
} hc_bfs_stats;

/* BFS from each source in turn (one persistent launch per source).
 * depth_out / parent_out: [num_sources][num_nodes] int32, -1 = unreached;
 * parent[src] = src.  Either may be NULL.  Replaces bfs_gpu
 * (src/kernels/gpu/bfs.cuh:21-95), which is bottom-up only and returns
 * parents alone. */
hc_status hc_bfs(hc_graph *g, const int32_t *sources, int32_t num_sources,
                 int32_t *depth_out, int32_t *parent_out,
                 const hc_bfs_opts *opts, hc_bfs_stats *stats);

/* No counterpart in the reference.  BFS from one source that allocates no
 * memory: for callers that cannot call cudaMalloc at that point -- code running
 * inside another framework's memory pool, paths that must avoid the device
 * synchronisation an allocation can cause, hosts that budget every byte of
 * HBM themselves.  index / neighbors / depth_out / parent_out are device
 * pointers of the current device ([num_nodes] int32 outputs, as hc_bfs).
 * The working set lives in a fixed device array inside the library (about
 * 13 MB, held by every GPU that loads it until exit), so graphs are limited to
 * 2^20 vertices and 2^24 edges; larger ones return HC_ERR_INVALID_ARG.
 * The first call on a device resolves that array's address (make it before
 * any stream capture).  All calls share the array: calls that overlap on the
 * GPU (other streams, other host threads) race and must not be issued.
 * Runs on `stream` (a cudaStream_t, NULL = legacy default) and returns after
 * the run has finished.  Before the traversal a check pass (its flag also in
 * the fixed array) refuses, with HC_ERR_INVALID_ARG, offsets that do not
 * rise from 0 to num_edges and neighbour ids outside [0, num_nodes).  It
 * uses Beamer's fixed alpha = 15 / beta = 18 and thread-per-vertex bottom-up
 * levels over every vertex (no degree analysis, no tuned values), so it can
 * be slower than hc_bfs on the same graph. */
hc_status hc_bfs_noalloc(const int64_t *index, const int32_t *neighbors, int32_t num_nodes,
                         int64_t num_edges, int32_t source, int32_t *depth_out,
                         int32_t *parent_out, void *stream);

/* ------------------------------------------------------------------ SSSP */

typedef struct hc_sssp_opts {
    int32_t delta;        /* near/far split width; 0 = auto, < 0 = plain frontier Bellman-Ford */
    int32_t max_epochs;   /* 0 = unlimited */
    int32_t collect_stats;
    int32_t pull_alpha;   /* run an epoch as a pull sweep over every row (the reference's
                             Bellman-Ford epoch, src/kernels/gpu/sssp.cuh:120-281) when the
                             frontier's edges * pull_alpha > M; 0 = auto (10), < 0 = never.
                             Needs symmetric weights (checked once per graph). */
} hc_sssp_opts;

typedef struct hc_sssp_stats {
    int32_t epochs;
    int32_t reached;
    int64_t vertices_processed;
    int64_t edges_relaxed;
    double bytes_model;
    double ms;
} hc_sssp_stats;

/* Single-source shortest paths over int32 weights (graph wtype HC_W_I32).
 * dist_out: [num_sources][num_nodes] int32, INT32_MAX = unreachable.
 * Distances are int32 and every candidate dist + w is clamped at INT32_MAX:
 * when a path of num_active - 1 edges of the largest weight could reach the
 * clamp, each source's distances are checked after its run, and a finite
 * distance within the largest weight of INT32_MAX (where a clamped candidate
 * could have hidden a longer one) returns HC_ERR_UNSUPPORTED.  The
 * reference's float distances lose integer exactness above 2^24 instead
 * (src/kernels/gpu/sssp.cuh:120-281).  hc_sssp_batched checks its 32-bit
 * groups the same way.
 * parent_out (optional): a shortest-path tree, parent[src] = src.
 * With pull epochs enabled the first call builds, and the handle keeps, a
 * second copy of the adjacency for the pull sweeps: each row's (neighbour,
 * weight) pairs ordered by weight, 8 * (num_edges + 64) bytes.  When a later
 * call of another kind cannot allocate what it needs, that copy (like the
 * other arrays a handle derives and can rebuild) is released and built
 * again by the next hc_sssp.
 * Replaces sssp_pull_gpu (src/kernels/gpu/sssp.cuh:42-100). */
hc_status hc_sssp(hc_graph *g, const int32_t *sources, int32_t num_sources,
                  int32_t *dist_out, int32_t *parent_out,
                  const hc_sssp_opts *opts, hc_sssp_stats *stats);

/* -------------------------------------------------------------- PageRank */

typedef struct hc_pr_opts {
    float damping;        /* 0 -> 0.85 (src/kernels/gpu/pr.cuh:149) */
    float tol_l1;         /* stop when sum |x_new - x_old| < tol_l1 (0 -> off) */
    float eps_vertex;     /* stop when no |x_new - x_old| > eps_vertex (0 -> off) */
    int32_t max_iters;    /* 0 -> 50 */
    int32_t weighted;     /* 1: transition weight w_uv / sum_k w_uk; 0: 1/deg(u) */
    hc_variant variant;
    int32_t accel;        /* when the walk is reversible (symmetric weights, or symmetric
                             structure unweighted): 0: adjoint by preconditioned conjugate
                             gradients, forward by Jacobi sweeps; 1: as 0, and Chebyshev
                             semi-iteration for the forward; 2: Chebyshev for the adjoint;
                             -1: Jacobi sweeps everywhere.  Other graphs: Jacobi sweeps. */
} hc_pr_opts;

typedef struct hc_pr_stats {
    int32_t iterations;
    int32_t converged;
    float residual_l1;
    int32_t changed;      /* vertices with |delta| > eps_vertex in the last iteration */
    double bytes_model;
    double ms;
} hc_pr_stats;

/* Pull PageRank, x = (1-d) t + d A x with A[v,u] = transition weight u->v,
 * no dangling redistribution (src/kernels/gpu/pr.cuh:140-174).  teleport:
 * [num_nodes][ncols] fp32 or NULL for uniform 1/N (ncols must be 1 then).
 * scores_out: [num_nodes][ncols] fp32.  ncols > 1 runs personalised
 * PageRank for all columns in one SpMM-form launch per iteration. */
hc_status hc_pr_forward(hc_graph *g, const float *teleport, int32_t ncols,
                        float *scores_out, const hc_pr_opts *opts,
                        hc_pr_stats *stats);

/* PageRank in the reference's own sweep order: scores updated in place from
 * vertex 0 to N-1, each vertex reading this sweep's scores of lower
 * neighbours and the previous sweep's of higher ones, a score stored only
 * when it moves by more than eps_vertex, until a sweep stores nothing (or
 * max_iters sweeps).  This is pr_pull_cpu with epoch_pr_pull_cpu_one_to_one
 * on one thread (src/kernels/cpu/pr.cuh:33-65, :157-187), and the rule of
 * pr_pull_gpu's epoch kernels (src/kernels/gpu/pr.cuh:42-118, :140-174)
 * without their run-to-run variation: the output equals the reference's
 * single-thread scores bit for bit.  Runs as a level schedule (built once per
 * graph) on the device; needs every edge to have a reverse
 * (HC_ERR_UNSUPPORTED otherwise).  init_scores: [num_nodes] fp32 or NULL for
 * 1/N.  opts: damping (0 -> 0.85), eps_vertex (0 -> 5e-8), max_iters (0 ->
 * no cap); tol_l1, weighted, variant and accel are ignored (unweighted
 * degrees, as the reference).  stats->iterations = sweeps, converged = 1 when
 * the last sweep stored nothing, changed = scores stored by the last sweep. */
hc_status hc_pr_pull_ordered(hc_graph *g, const float *init_scores, float *scores_out,
                             const hc_pr_opts *opts, hc_pr_stats *stats);

/* Adjoint of hc_pr_forward for ncols == 1.  Given the converged scores x and
 * dL/dx, solves lambda = dL/dx + d A^T lambda and returns
 * dL/dteleport = (1-d) lambda and, if dL_dweights != NULL, the gradient
 * with respect to the raw edge weights (CSR slot order; unit weights when the
 * graph is unweighted), chained through the row normalisation.
 * Here opts->tol_l1 is relative: the solve stops when sum |lambda_new -
 * lambda_old| < tol_l1 * sum |dL/dx|.
 * No counterpart in the reference. */
hc_status hc_pr_backward(hc_graph *g, const float *scores, const float *dL_dscores,
                         float *dL_dteleport, float *dL_dweights,
                         const hc_pr_opts *opts, hc_pr_stats *stats);

/* Personalised PageRank for ncols teleport vectors at once (SpMM form):
 * column c teleports uniformly to seeds[seed_offsets[c] .. seed_offsets[c+1]).
 * scores_out: [num_nodes][ncols] fp32, 1 <= ncols <= 256.  Iterates until
 * every column's L1 change is below tol_l1 or max_iters.
 * No counterpart in the reference (it runs one uniform PageRank per call). */
hc_status hc_ppr_batched(hc_graph *g, const int32_t *seed_offsets, const int32_t *seeds,
                         int32_t ncols, float *scores_out, const hc_pr_opts *opts,
                         hc_pr_stats *stats);

/* --------------------------------------------------------------- batched */

/* hc_batch_opts.use_graph */
#define HC_GRAPH_AUTO 0   /* the library's choice (a graph where the loop has one) */
#define HC_GRAPH_ON 1     /* run the epoch loop as a CUDA graph (while node) */
#define HC_GRAPH_OFF 2    /* host loop: one launch sequence and one sync per epoch */

typedef struct hc_batch_opts {
    int32_t group;        /* sources per group (0 = tuned, else sized to free memory) */
    int32_t max_epochs;   /* 0 = unlimited */
    int32_t use_graph;    /* HC_GRAPH_AUTO / _ON / _OFF */
    int32_t switch_alpha; /* direction switch (0 = tuned / default, < 0 = never switch):
                             BFS pushes while frontier edges * alpha < M (default 10),
                             else pulls; < 0 pulls every level.  SSSP pulls when the
                             queue's edges * alpha > M (default 2); < 0 pushes only. */
    int32_t dist_bits;    /* batched SSSP working distances: 0 = 16-bit when every weight
                             is at most 4095 (a group whose distances do not fit runs
                             again 32-bit), 16 = the same, 32 = always 32-bit.  The
                             output is int32 either way. */
} hc_batch_opts;

typedef struct hc_batch_stats {
    int32_t epochs;
    int32_t groups;
    double bytes_model;
    double ms;
    int32_t wide_groups;  /* batched SSSP: groups run with 32-bit distances */
    int32_t reruns;       /* batched SSSP: 16-bit groups run again 32-bit */
} hc_batch_stats;

/* Multi-source BFS: bit-sliced frontiers, all sources of a group advance in
 * one launch per level.  depth_out: [num_sources][num_nodes] int32.
 * The reference runs sources one after another (src/benchmarks/gpu_benchmark.cuh:577-586). */
hc_status hc_bfs_batched(hc_graph *g, const int32_t *sources, int32_t num_sources,
                         int32_t *depth_out, const hc_batch_opts *opts,
                         hc_batch_stats *stats);

/* Multi-source SSSP, one lane per source over vertex-major distances.
 * dist_out: [num_sources][num_nodes] int32. */
hc_status hc_sssp_batched(hc_graph *g, const int32_t *sources, int32_t num_sources,
                          int32_t *dist_out, const hc_batch_opts *opts,
                          hc_batch_stats *stats);

/* ------------------------------------------------------------- autotuner */

/* Launch parameters of one graph, picked by hc_autotune.  A zero field in an
 * opts struct (hc_bfs_opts.alpha, hc_sssp_opts.delta, hc_batch_opts.group ...)
 * means "the tuned value", or the built-in default while a field is untuned
 * (zero here).  No counterpart in the reference, whose variant and launch
 * shape are chosen by hand per call (src/kernels/gpu/bfs.cuh:352-360). */
#define HC_BFS_SPLIT_LEVELS 8
typedef struct hc_tuning {
    int32_t bfs_alpha;          /* hc_bfs_opts.alpha */
    int32_t bfs_beta;           /* hc_bfs_opts.beta */
    int32_t bfs_bu_variant;     /* hc_bfs_opts.bu_variant (HC_VARIANT_AUTO = untuned) */
    int32_t sssp_delta;         /* hc_sssp_opts.delta */
    int32_t sssp_pull_alpha;    /* hc_sssp_opts.pull_alpha */
    int32_t mbfs_group;         /* hc_bfs_batched group */
    int32_t mbfs_switch_alpha;  /* hc_bfs_batched switch_alpha */
    int32_t mssp_group;         /* hc_sssp_batched group */
    int32_t mssp_switch_alpha;  /* hc_sssp_batched switch_alpha */
    int32_t trials;             /* candidates timed by the last hc_autotune */
    double tune_ms;             /* device time spent on them */
    /* Per bottom-up BFS level granularity (HC_TUNE_BFS_LEVELS): bottom-up
     * level k (0 = the first of a run) visits vertices [0, bfs_bu_split[k])
     * warp per vertex and the rest thread per vertex (later levels use the
     * last entry).  Used by hc_bfs when hc_bfs_opts.bu_variant is AUTO and
     * bfs_bu_split_levels > 0; the candidates are equal-edge segment bounds
     * (hc_equal_edge_ranges), 32-aligned. */
    int32_t bfs_bu_split[HC_BFS_SPLIT_LEVELS];
    int32_t bfs_bu_split_levels;
    /* Blocks per SM of the persistent SSSP kernel (its push epochs): fewer
     * blocks make each grid barrier cheaper, more give large frontiers more
     * warps.  0 = as many as fit (2). */
    int32_t sssp_blocks_per_sm;
} hc_tuning;

#define HC_TUNE_BFS 1u
#define HC_TUNE_SSSP 2u
#define HC_TUNE_BFS_BATCHED 4u
#define HC_TUNE_SSSP_BATCHED 8u
#define HC_TUNE_BFS_LEVELS 16u
#define HC_TUNE_ALL 31u

/* Times candidate parameters on the sample sources (CUDA events, outputs
 * discarded) by coordinate descent, one parameter at a time from the current
 * values, and stores the fastest on the handle; `out` (optional) receives the
 * result.  The batched searches run on up to 256 / 512 of the samples. */
hc_status hc_autotune(hc_graph *g, const int32_t *sample_sources, int32_t num_samples,
                      uint32_t what, hc_tuning *out);
/* Reads / replaces the handle's tuning (e.g. one saved from an earlier run). */
hc_status hc_get_tuning(const hc_graph *g, hc_tuning *out);
hc_status hc_set_tuning(hc_graph *g, const hc_tuning *t);

/* ------------------------------------------------------ device memory */
/* Plain device-memory helpers so hosts that drive the epoch kernels below
 * need no CUDA headers.  Replace the cudaMalloc / cudaMemcpy / cudaMemset /
 * cudaFree calls of the reference drivers (src/kernels/gpu/sssp.cuh:52-97,
 * src/bitmap.cuh:192-226). */
hc_status hc_dev_malloc(void **ptr, size_t bytes, int32_t device);
hc_status hc_dev_free(void *ptr);
hc_status hc_memcpy(void *dst, const void *src, size_t bytes); /* any direction, synchronous */
hc_status hc_dev_memset(void *ptr, int32_t value, size_t bytes);
hc_status hc_device_synchronize(void);
/* Kernels launched by this library in this process so far. */
int64_t hc_kernel_launches(void);

/* ------------------------------------------------- segment profiling */
/* Vertex ranges of about equal edge count, the reference's
 * compute_equal_edge_ranges (src/graph.cuh:156-201): walking the vertices in
 * order, a segment closes at the vertex whose degree brings its running sum to
 * at least num_edges / num_segments (that vertex opens the next one); the
 * last segment ends at num_nodes, and inner bounds are rounded to the nearest
 * multiple of chunk_size.  ranges_out: num_segments + 1 entries.  Three
 * departures keep every vertex in exactly one segment where the reference
 * does not: closures past num_segments - 1 are dropped (the reference writes
 * past its array when the edge total is not divisible by the count, or is
 * below it), the last segment always ends at num_nodes (the reference's ends
 * at the vertex that closed it when num_segments closures happen), and bounds
 * never round past num_nodes.  index: host array. */
hc_status hc_equal_edge_ranges(const int64_t *index, int32_t num_nodes, int32_t num_segments,
                               int32_t chunk_size, int32_t *ranges_out);

typedef enum hc_profile_algo {
    HC_PROFILE_SSSP = 0,  /* epoch_sssp_pull_gpu_* (hc_epoch_sssp_pull) */
    HC_PROFILE_PR = 1,    /* epoch_pr_pull_gpu_* (hc_epoch_pr_pull) */
    HC_PROFILE_BFS = 2    /* epoch_bfs_pull_gpu_* / sync warp (hc_epoch_bfs_pull / _sync_pull) */
} hc_profile_algo;

/* segment_res_t (src/benchmarks/benchmark.cuh:36-47). */
typedef struct hc_segment_result {
    int32_t start_id, end_id;  /* [start_id, end_id) */
    int64_t num_edges;
    float avg_degree, min_degree, max_degree;
    int32_t epoch;             /* BFS: the level profiled; -1 otherwise */
    double millis;             /* mean over `iters` launches */
    double gteps;              /* num_edges / 2 per second, the reference's formula */
} hc_segment_result;

/* The per-segment benchmark of the reference's TreeBenchmark
 * (src/benchmarks/benchmark.cuh:87-309, gpu_benchmark.cuh:201-330): for each
 * segment [ranges[s], ranges[s+1]) one epoch kernel launch of `variant`
 * (sync_iters > 0: the sync-warp BFS kernel) with the given shape, timed with
 * CUDA events over `iters` launches from the same initial state (SSSP / PR: a
 * seeded random vector; BFS: the state before level `level` of a BFS from
 * `source`).  out: num_segments results. */
hc_status hc_profile_segments(hc_graph *g, hc_profile_algo algo, hc_variant variant, int32_t sync_iters,
                              const int32_t *ranges, int32_t num_segments, int32_t source, int32_t level,
                              int32_t block_count, int32_t thread_count, int32_t iters,
                              hc_segment_result *out);

/* ------------------------------------------------------- time limits */
/* No counterpart in the reference, whose host loops wait without a bound.
 * Every device-side wait here is bounded: a grid barrier gives up after
 * wait_ns (default 2 s), one persistent run after run_ns (20 s), one batched
 * group's epoch loop after loop_ns (60 s); each then ends its call with
 * HC_ERR_TIMEOUT and leaves the handle usable.  hc_set_time_limits replaces
 * the three bounds on `device` for every later launch in this process
 * (0 = the default); it exists so that tests can make each wait run out. */
hc_status hc_set_time_limits(int32_t device, uint64_t wait_ns, uint64_t run_ns, uint64_t loop_ns);
/* Runs the grid barrier alone on `device` with `blocks` (1..64) co-resident
 * blocks, block `withhold_block` never arriving (-1: all arrive), and returns
 * the barrier's recorded status in *status_out: HC_OK when all arrived,
 * HC_ERR_TIMEOUT when the others gave up after the wait limit. */
hc_status hc_selftest_grid_barrier(int32_t device, int32_t blocks, int32_t withhold_block,
                                   int32_t *status_out);

/* ------------------------------------------------ reference epoch kernels */
/* One epoch of the reference's in-place pull kernels over [start_id, end_id),
 * device pointers only, launched on `stream` with the given shape and
 * granularity, adding to *updated (device int32).  These keep the epoch-kernel
 * contract of src/kernels/kernel_types.cuh:36-63 for callers that drive their
 * own epoch loop.  Like the reference's kernels they trust the CSR they are
 * given (the contract carries no vertex or edge count to check against, and a
 * per-epoch pass would double each epoch's traffic): check it once with
 * hc_csr_check before the loop, as the reference-shaped drivers in
 * hc_compat.hpp do. */

/* epoch_bfs_sync_pull_gpu_warp<sync_iters> (src/kernels/gpu/bfs.cuh:234-288):
 * the warp-per-vertex bottom-up epoch that probes sync_iters (>= 1) 32-edge
 * chunks of a row before the warp votes.  Same arguments as hc_epoch_bfs_pull;
 * thread_count a multiple of 32. */
hc_status hc_epoch_bfs_sync_pull(const int64_t *index, const int32_t *neighbors,
                                 int32_t *parents, int32_t start_id, int32_t end_id,
                                 const uint32_t *frontier, uint32_t *next_frontier,
                                 int32_t *num_nodes, int32_t sync_iters,
                                 int32_t block_count, int32_t thread_count, void *stream);

/* Checks a CSR in device memory: offsets rising from index[0] == 0 to
 * index[num_nodes] == num_edges and every neighbour id in [0, num_nodes);
 * HC_ERR_INVALID_ARG otherwise.  `neighbors` holds num_edges int32 ids, or,
 * with interleaved = 1, the reference's {int32 v; float w} wnode_t array
 * (src/graph.cuh:37-41).  One pass on `stream`; returns when it is done.
 * Replaces nothing in the reference, whose drivers upload without a check
 * (src/kernels/gpu/sssp.cuh:51-61). */
hc_status hc_csr_check(const int64_t *index, const void *neighbors, int32_t interleaved,
                       int32_t num_nodes, int64_t num_edges, void *stream);

/* sssp_gpu_epoch_func (src/kernels/kernel_types.cuh:36-37): wnodes is the
 * reference's interleaved {int32 v; float w} edge array. */
hc_status hc_epoch_sssp_pull(const int64_t *index, const void *wnodes,
                             int32_t start_id, int32_t end_id, float *dist,
                             int32_t *updated, hc_variant variant,
                             int32_t block_count, int32_t thread_count,
                             void *stream);

/* pr_gpu_epoch_func (src/kernels/kernel_types.cuh:46-47). */
hc_status hc_epoch_pr_pull(const int64_t *index, const void *wnodes,
                           int32_t start_id, int32_t end_id, float *score,
                           int32_t *updated, int32_t num_nodes,
                           const int64_t *degrees, hc_variant variant,
                           int32_t block_count, int32_t thread_count,
                           void *stream);

/* bfs_gpu_epoch_func (src/kernels/kernel_types.cuh:60-63): the Bitmap
 * structs become their 32-bit word buffers. */
hc_status hc_epoch_bfs_pull(const int64_t *index, const int32_t *neighbors,
                            int32_t *parents, int32_t start_id, int32_t end_id,
                            const uint32_t *frontier, uint32_t *next_frontier,
                            int32_t *num_nodes, hc_variant variant,
                            int32_t block_count, int32_t thread_count,
                            void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HC_H */
