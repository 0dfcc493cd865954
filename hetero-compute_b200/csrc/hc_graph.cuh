// The device graph handle shared by every kernel translation unit.
#pragma once

#include "hc_device.cuh"

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
    int32_t max_degree = 0;
    hc_wtype wtype = HC_W_NONE;

    hc::DevBuf index, nbr, wgt;

    // lazily built derived data
    hc::DevBuf inv_deg;        // f32[N]: 1/deg (0 for isolated)
    hc::DevBuf inv_wsum;       // f32[N]: 1/sum_k w_uk (weighted PageRank)
    hc::DevBuf wtn;            // f32[M]: slot (v,i) holds w_{u v}/sum_k w_uk, u = nbr[v][i]
    hc::DevBuf pr_plan;        // PageRank row blocks
    int32_t pr_plan_blocks = 0;
    int32_t pr_plan_tasks = 0;
    int32_t pr_plan_huge = 0;
    hc::DevBuf pr_plan_huge_rows;

    // workspaces
    hc::DevBuf ws_bfs, ws_sssp, ws_pr, ws_batch, ws_out0, ws_out1, ws_ctl;
    hc::PinnedBuf pinned;

    int bfs_grid = 0, sssp_grid = 0;
    int64_t bytes_held() const;
};

namespace hc {
// Make the handle's device current; returns HC_ERR_CUDA on failure.
hc_status activate(hc_graph *g);
// Builds inv_deg (and, for weighted graphs, inv_wsum / wtn) if missing.
hc_status ensure_pr_derived(hc_graph *g, bool weighted);
}  // namespace hc
