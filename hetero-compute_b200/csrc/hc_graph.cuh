// The device graph handle shared by every kernel translation unit.
#pragma once

#include "hc_device.cuh"

namespace hc {
// Row plan shared by the PageRank sweeps and the SSSP pull sweep, built once
// per graph from the offsets of the rows with edges:
//   stream groups  32 consecutive rows with <= kStreamEdges edges in total
//   long rows      <= kHubEdges edges, one warp per row
//   hub rows       > kHubEdges edges, cut into kHubChunk-edge tasks
constexpr int kStreamEdges = 2048;
constexpr int kHubEdges = 4096;
constexpr int kHubChunk = 2048;
// Batched SSSP keeps 16-bit distances when no weight exceeds this.
constexpr int32_t kMsspNarrowMaxW = 0x0FFF;

struct HubInfo {
    int32_t row;
    int32_t first;  // first partial slot
    int32_t nchunks;
    int32_t pad;
};

struct PrPlanDev {
    const int32_t *stream;  // group ids (rows 32*id .. 32*id+31)
    const int32_t *longrows;
    const int2 *tasks;      // (hub index, chunk)
    const HubInfo *hubs;
    int n_stream, n_long, n_tasks, n_hub;
};
}  // namespace hc

// Layout in HBM (one allocation per array, 256-byte aligned by cudaMalloc):
//   index     int64[N+1]                 row offsets
//   nbr       int32[M + kNbrPad]         neighbours; the pad keeps 128-bit
//                                        loads of a row's last aligned window
//                                        inside the allocation
//   wgt       int32/f32[M + kNbrPad]     weights, same slots as nbr (SoA)
// Derived arrays (inverse degrees, transposed weights, PageRank row plan)
// and per-algorithm workspaces are built lazily and kept with the handle.
struct hc_graph {
    int device = 0;
    int sm_count = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;

    int32_t N = 0;
    int64_t M = 0;
    int32_t n_active = 0;      // vertices [0, n_active) may have edges
    int32_t n_warp_rows = 0;   // degree-sorted: [0, n_warp_rows) have degree >= 32 (32-aligned)
    int32_t degree_sorted = 0;
    int32_t rows_sorted = 0;      // every row strictly increasing
    int32_t max_degree = 0;
    hc_wtype wtype = HC_W_NONE;

    hc::DevBuf index, nbr, wgt;

    // lazily built derived data
    hc::DevBuf inv_deg;        // f32[N]: 1/deg (0 for isolated)
    hc::DevBuf inv_wsum;       // f32[N]: 1/sum_k w_uk (weighted PageRank)
    hc::DevBuf wtn;            // f32[M]: slot (v,i) holds w_{u v}/sum_k w_uk, u = nbr[v][i]
    hc::DevBuf wf32;           // f32[M]: int32 weights as floats (weighted PageRank on int32 graphs)
    hc::DevBuf pr_plan;        // row plan (device arrays)
    hc::PrPlanDev pr_view{};   // host copy of its pointers and counts
    int32_t pr_partial_slots = 0;
    hc::DevBuf pr_plan_huge_rows;
    // level schedule of the reference-order PageRank sweep (hc_pr_ordered.cu):
    // order[N] | level_off[levels + 1] | level_long[levels] | deg as fp32 [N];
    // levels -1 = not built
    hc::DevBuf pr_ord;
    int32_t pr_ord_levels = -1;

    // symmetry of the PageRank transition (-1: not checked yet)
    int pr_sym_struct = -1;    // every edge u->v has v->u (rows sorted)
    int pr_sym_w = -1;         // ... with the same weight

    // weight statistics, computed once
    int wstats_done = 0;
    int w_negative = 0;
    int32_t w_max = 0;         // largest weight (0 when none is positive)
    double w_mean = 0.0;
    int w_symmetric = 0;       // w(u->v) == w(v->u) for every edge (rows sorted)
    // SSSP pull sweeps: int2[M + 64] (neighbour, weight) pairs of each row in
    // weight-bucket order (stable), built on the first pull-enabled call
    hc::DevBuf sssp_adj;
    int sssp_adj_ready = 0;

    // batched-BFS hub plan (rows above its split threshold, (row, chunk) tasks)
    hc::DevBuf ws_plan_ms;
    int32_t ms_hubs = -1, ms_tasks = 0;
    // batched-SSSP pull plan: (row, chunk) tasks of the rows above its chunk size
    hc::DevBuf ws_plan_mssp;
    int32_t mssp_tasks = -1;
    int32_t mssp_hub_rows = -1;  // degree-sorted: the row prefix holding half the edges

    // autotuned launch parameters (zero fields: built-in defaults)
    hc_tuning tune{};

    // host-output pipeline (per-source results copied while the next computes)
    hc::DevBuf ws_stage[2][2];  // [slot][array]
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_ready[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr};

    // workspaces
    hc::DevBuf ws_bfs, ws_sssp, ws_pr, ws_batch, ws_out0, ws_out1, ws_ctl, ws_src;
    hc::PinnedBuf pinned;
    // mapped pinned slots for control-block reads (ctl_read), and their device address
    void *ctl_host = nullptr;
    void *ctl_host_dev = nullptr;

    int bfs_grid = 0, sssp_grid = 0;
    int64_t bytes_held() const;
};

namespace hc {
// Make the handle's device current; returns HC_ERR_CUDA on failure.
hc_status activate(hc_graph *g);
// Builds inv_deg (and, for weighted graphs, inv_wsum / wtn) if missing.
hc_status ensure_pr_derived(hc_graph *g, bool weighted);
// Per-source outputs bound for host memory, double-buffered: source i writes
// staging slot i & 1 on the compute stream, and its copy to the caller runs
// on a copy stream while the next source computes (overlapped when the
// destination is pinned).  Before a slot is written again the compute stream
// waits for that slot's previous copy.
struct OutPipe {
    hc_graph *g = nullptr;
    int narr = 0;
    size_t bytes = 0;
    size_t copy_bytes = 0;  // bytes of each array copied out (init: all; a caller may shorten it)
    bool pending = false;
    int pend_slot = 0;
    void *pend_dst[2] = {nullptr, nullptr};
    // Staging and events for `arrays` outputs of `bytes` each.
    hc_status init(hc_graph *graph, int arrays, size_t each);
    // Staging buffers of source i (after the wait for the slot's last copy).
    hc_status acquire(int i, int32_t **bufs);
    // Source i's results are complete on the compute stream once what is
    // queued there has run; copy them to dst[] (null entries are skipped).
    // The copy is issued by the next acquire or by finish.
    hc_status release(int i, void *const *dst);
    hc_status flush();
    hc_status finish();
};

// A handle for an N-vertex, M-edge graph on `device` with its CSR arrays
// allocated (neighbour and weight pads zeroed) and not yet filled.
hc_status graph_alloc(int32_t num_nodes, int64_t num_edges, hc_wtype wtype, int32_t device, hc_graph **out);
// Validates the filled CSR (offsets 0..M non-decreasing, ids in [0, N)) and
// records its degree analysis; `who` names the caller in error messages.
hc_status graph_finish(hc_graph *g, const char *who);
// Checks a caller's CSR on the device (offsets rising from 0 to m, neighbour
// ids in [0, n); `stride` 2 for interleaved {id, weight} edges): clears
// *flag_dev, then sets bit 0 (offsets) / bit 1 (ids) on a violation.
hc_status csr_check_async(const int64_t *index, const int32_t *nbr, int stride, int32_t n, int64_t m, int *flag_dev,
                          int sm_count, cudaStream_t s);
// Whether the PageRank transition is a reversible walk (symmetric structure,
// and symmetric weights when `weighted`), checked once per graph.
hc_status ensure_pr_symmetry(hc_graph *g, bool weighted, bool *symmetric);
// Whether every edge u->v has a reverse v->u (as multisets), and whether the
// reverse carries the same weight bits (`wbits` may be null).
hc_status edge_symmetry(hc_graph *g, const uint32_t *wbits, bool *structure, bool *weights);
// The edge weights as fp32 for weighted PageRank: the weight array itself
// (fp32 graphs) or its converted copy (int32 graphs, built by ensure_pr_derived).
const float *pr_weights(const hc_graph *g);
// Builds the row plan if missing (g->pr_view, g->pr_partial_slots).
hc_status ensure_plan(hc_graph *g);
// Computes w_negative, w_max, w_mean and w_symmetric once (int32 weights).
hc_status ensure_weight_stats(hc_graph *g);
// Per-run control traffic kept off the copy engines.  A host-output call
// keeps a large copy on the copy stream while the next source runs; a small
// cudaMemcpyAsync or cudaMemsetAsync of a control block on the compute stream
// can queue on the same engine behind it and serialise the two.  ctl_zero
// clears device words with a one-block kernel on the graph's stream; ctl_read
// has a one-block kernel write `bytes` (at most kCtlSlotBytes) of device memory
// into mapped pinned slot `slot` (0..kCtlSlots-1) and returns its host address,
// valid once the stream has been synchronised.
constexpr size_t kCtlSlotBytes = 4096;
constexpr int kCtlSlots = 4;
hc_status ctl_zero(hc_graph *g, void *dev, size_t bytes);
hc_status ctl_read(hc_graph *g, const void *dev, size_t bytes, int slot, const void **host);
// Device memory pressure.  Derived arrays that can be built again (the
// pull sweeps' pair array, the reference-order schedule, the weighted
// PageRank arrays) and the batched workspace are released, when an
// allocation fails, unless the running call needs them; the allocation is
// then tried once more.  A call states what it needs for its lifetime.
enum : unsigned { kKeepAdj = 1u, kKeepPrOrd = 2u, kKeepPrWeighted = 4u, kKeepBatch = 8u };
struct ReclaimScope {
    ReclaimScope(hc_graph *g, unsigned keep);
    ~ReclaimScope();
    ReclaimScope(const ReclaimScope &) = delete;
    ReclaimScope &operator=(const ReclaimScope &) = delete;
    hc_graph *prev_g;
    unsigned prev_keep;
};
// The pull sweeps' weight-ordered (neighbour, weight) pairs (hc_graph::sssp_adj),
// after the weight statistics; bucket(w) = w >> weight_shift(w_max) < 256.
hc_status ensure_weight_order(hc_graph *g);
int weight_shift(int32_t w_max);
}  // namespace hc
