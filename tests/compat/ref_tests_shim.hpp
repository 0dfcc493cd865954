// TEST INFRASTRUCTURE: builds the reference's own test programs
// (tests/{bfs,sssp,pr}/*_verify.cu of chrisliu/hetero-compute), unchanged,
// against this library's drop-in header.  Force-included ahead of a test
// source (nvcc -include), it claims the include guards of the reference's GPU
// and heterogeneous driver headers, its graph / bitmap / kernel-type headers,
// so that those come from include/hc_compat.hpp instead; the reference's CPU
// kernels (src/kernels/cpu/*.cuh, its oracle in these tests), util.h and
// window.h still compile from its own tree.  Only the CPU epoch-function
// typedefs of src/kernels/kernel_types.cuh:29-68 are restated here, since
// that header is claimed whole.
#pragma once

#define SRC__GRAPH_CUH
#define SRC__BITMAP_CUH
#define SRC_KERNELS__KERNEL_TYPES_CUH
#define SRC_KERNELS_GPU__KERNEL_SSSP_CUH
#define SRC_KERNELS_GPU__KERNEL_PR_CUH
#define SRC_KERNELS_GPU__BFS_CUH
#define SRC_KERNELS_HETEROGENEOUS__SSSP_CUH
#define SRC_KERNELS_HETEROGENEOUS__PR_CUH
#define SRC_KERNELS_HETEROGENEOUS__BFS_CUH

#include "hc_compat.hpp"
#include "src/window.h"

typedef void (*sssp_cpu_epoch_func)(const CSRWGraph &, weight_t *, const nid_t, const nid_t, const int, const int,
                                    nid_t &);
typedef void (*pr_cpu_epoch_func)(const CSRWGraph &, weight_t *, const nid_t, const nid_t, const int, const int,
                                  nid_t &);
typedef void (*bfs_cpu_push_epoch_func)(const CSRUWGraph &, nid_t *const, SlidingWindow<nid_t> &, nid_t &);
typedef void (*bfs_cpu_pull_epoch_func)(const CSRUWGraph &, nid_t *const, const nid_t, const nid_t,
                                        const Bitmap::Bitmap *const, Bitmap::Bitmap *const, nid_t &);
typedef double(bfs_cpu_kernel)(const CSRUWGraph &g, const nid_t, nid_t **const);
