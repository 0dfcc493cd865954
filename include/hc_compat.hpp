// hc_compat.hpp -- the reference's host-side GPU API, re-exposed over the C ABI.
//
// Code written against chrisliu/hetero-compute's GPU drivers keeps its
// spelling: the graph types and loader (src/graph.cuh:26-239), SourcePicker
// (src/graph.cuh:106-141), the epoch-kernel registries BFSGPU / SSSPGPU /
// PRGPU with get_kernel / get_kernels / to_string / to_repr
// (src/kernels/gpu/bfs.cuh:295-365, src/kernels/gpu/sssp.cuh:287-356,
// src/kernels/gpu/pr.cuh:324-393) and the drivers bfs_gpu / sssp_pull_gpu /
// pr_pull_gpu (src/kernels/gpu/bfs.cuh:21-95, src/kernels/gpu/sssp.cuh:42-100,
// src/kernels/gpu/pr.cuh:42-118), with the same argument meaning, ownership
// (results returned as new[] arrays the caller delete[]s) and return value
// (milliseconds of the epoch loop).
//
// An epoch-kernel "function pointer" here is a handle naming a granularity.
// The reference names (epoch_sssp_pull_gpu_warp_red, ...) run that
// granularity's in-place pull epochs in a host-driven loop, exactly like the
// reference drivers; the *_auto handles run this engine's device-driven
// paths (direction-optimising BFS, near/far SSSP, Jacobi PageRank).
// Errors keep the reference's behaviour: message on stderr, exit(EXIT_FAILURE)
// (src/cuda.cuh:14-21).
//
// Host C++ only: compile with any C++17 compiler and link libhc.so.
#pragma once

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <ostream>
#include <random>
#include <string>
#include <vector>

#include "hc.h"

using nid_t = std::int32_t;
using weight_t = float;
using offset_t = std::int64_t;

const weight_t INF_WEIGHT = std::numeric_limits<weight_t>::infinity();
const nid_t INVALID_NODE = -1;

struct wnode_t {
    nid_t v;
    weight_t w;
};

namespace hc_compat {
inline void check(hc_status s, const char *what);
}
inline void hc_compat_dev_alloc(void **p, size_t bytes);
namespace hc_compat {
inline void check(hc_status s, const char *what) {
    if (s != HC_OK) {
        std::cerr << "[" << what << "] " << hc_status_string(s) << ": " << hc_last_error() << std::endl;
        std::exit(EXIT_FAILURE);
    }
}
template <class T>
inline nid_t target(const T &x);
template <>
inline nid_t target<nid_t>(const nid_t &x) { return x; }
template <>
inline nid_t target<wnode_t>(const wnode_t &x) { return x.v; }
}  // namespace hc_compat

inline void hc_compat_dev_alloc(void **p, size_t bytes) {
    hc_compat::check(hc_dev_malloc(p, bytes, 0), "hc_dev_malloc");
}

template <typename NeighborT>
class GenericCSRGraph {
public:
    offset_t *index = nullptr;
    NeighborT *neighbors = nullptr;
    nid_t num_nodes = 0;
    offset_t num_edges = 0;

    GenericCSRGraph() = default;
    GenericCSRGraph(const GenericCSRGraph &) = delete;
    GenericCSRGraph &operator=(const GenericCSRGraph &) = delete;
    GenericCSRGraph(GenericCSRGraph &&o) noexcept { *this = std::move(o); }
    GenericCSRGraph &operator=(GenericCSRGraph &&o) noexcept {
        std::swap(index, o.index);
        std::swap(neighbors, o.neighbors);
        std::swap(num_nodes, o.num_nodes);
        std::swap(num_edges, o.num_edges);
        return *this;
    }
    ~GenericCSRGraph() {
        delete[] index;
        delete[] neighbors;
    }
    // The range of nid's neighbours, iterable as the reference's
    // (src/graph.cuh:60-80: `for (wnode_t nei : g.get_neighbors(v))`).
    struct Neighborhood {
        const NeighborT *first, *last;
        const NeighborT *begin() const { return first; }
        const NeighborT *end() const { return last; }
    };
    Neighborhood get_neighbors(nid_t nid) const { return {neighbors + index[nid], neighbors + index[nid + 1]}; }
    offset_t get_degree(nid_t nid) const { return index[nid + 1] - index[nid]; }
    bool has_self_cycle(nid_t nid) const {
        for (offset_t i = index[nid]; i < index[nid + 1]; i++)
            if (hc_compat::target(neighbors[i]) == nid) return true;
        return false;
    }
};

using CSRWGraph = GenericCSRGraph<wnode_t>;
using CSRUWGraph = GenericCSRGraph<nid_t>;

// .sg / .wsg loader (src/graph.cuh:207-239), through hc_csr_read.
template <typename GraphT>
GraphT load_graph_from_file(const char *filename) {
    constexpr bool weighted = std::is_same<GraphT, CSRWGraph>::value;
    hc_csr c{};
    hc_compat::check(hc_csr_read(filename, weighted ? 1 : 0, &c), "load_graph_from_file");
    GraphT g;
    g.num_nodes = c.num_nodes;
    g.num_edges = c.num_edges;
    g.index = new offset_t[(size_t)c.num_nodes + 1];
    std::copy(c.index, c.index + c.num_nodes + 1, g.index);
    using N = typename std::remove_pointer<decltype(g.neighbors)>::type;
    g.neighbors = new N[(size_t)c.num_edges];
    for (offset_t i = 0; i < c.num_edges; i++) {
        if constexpr (weighted) g.neighbors[i] = wnode_t{c.neighbors[i], ((float *)c.weights)[i]};
        else g.neighbors[i] = c.neighbors[i];
    }
    hc_csr_free(&c);
    return g;
}

// SourcePicker (src/graph.cuh:106-141): the same draw sequence as
// hc_pick_sources, kept incrementally.
template <typename GraphT>
class SourcePicker {
public:
    explicit SourcePicker(const GraphT *g, nid_t const_source = -1)
        : g_(g), const_source_(const_source), rng_(37525), dist_(0, g->num_nodes - 1) {}
    nid_t next_vertex() {
        if (const_source_ >= 0) return const_source_;
        for (;;) {
            nid_t s = dist_(rng_);
            offset_t d = g_->get_degree(s);
            if (d == 0 || (d == 1 && g_->has_self_cycle(s))) continue;
            return s;
        }
    }
    void reset() { rng_.seed(37525); dist_.reset(); }

private:
    const GraphT *g_;
    nid_t const_source_;
    std::mt19937 rng_;
    std::uniform_int_distribution<nid_t> dist_;
};

// ----------------------------------------------------------------- Bitmap
// The reference's Bitmap (src/bitmap.cuh:14-191): the struct layout and the
// functions epoch kernels and drivers call.  Host functions are plain C++ over
// the C ABI's memory helpers; get_bit / set_bit are host-and-device and
// cu_set_bit_atomic device-only under nvcc, so epoch kernels a caller writes
// against the reference's API compile unchanged.
#ifdef __CUDACC__
#define HC_COMPAT_HD __host__ __device__
#else
#define HC_COMPAT_HD
#endif
namespace Bitmap {
using data_t = int;
const std::size_t data_size = sizeof(data_t) * 8;
HC_COMPAT_HD inline std::size_t data_offset(std::size_t n) { return n / data_size; }
HC_COMPAT_HD inline std::size_t bit_offset(std::size_t n) { return n & (data_size - 1); }
struct Bitmap {
    data_t *buffer;
    bool using_cuda;
    std::size_t size;  // words
};
HC_COMPAT_HD inline void set_bit(Bitmap *const b, const std::size_t idx) {
    b->buffer[data_offset(idx)] |= static_cast<data_t>(1) << bit_offset(idx);
}
HC_COMPAT_HD inline bool get_bit(const Bitmap *const b, const std::size_t idx) {
    return (b->buffer[data_offset(idx)] >> bit_offset(idx)) & static_cast<data_t>(1);
}
#ifdef __CUDACC__
__device__ inline void cu_set_bit_atomic(Bitmap *const b, const std::size_t idx) {
    atomicOr(b->buffer + data_offset(idx), static_cast<data_t>(1) << bit_offset(idx));
}
#endif
inline void set_bit_atomic(Bitmap *const b, const std::size_t idx) {
    __atomic_fetch_or(&b->buffer[data_offset(idx)], static_cast<data_t>(1) << bit_offset(idx), __ATOMIC_RELAXED);
}
inline void reset(Bitmap *const b) { std::fill(b->buffer, b->buffer + b->size, 0); }
inline bool copy(const Bitmap *const from, Bitmap *const to) {
    if (from->size != to->size) return false;
    std::copy(from->buffer, from->buffer + from->size, to->buffer);
    return true;
}
// Host bitmap (use_cuda: its buffer in device memory instead, as the
// reference's pinned-or-device variants are used by its drivers).
inline Bitmap *constructor(const std::size_t num_elements, const bool use_cuda = false) {
    Bitmap *b = new Bitmap{nullptr, use_cuda, (num_elements + data_size - 1) / data_size};
    if (use_cuda) {
        hc_compat_dev_alloc((void **)&b->buffer, b->size * sizeof(data_t));
        hc_dev_memset(b->buffer, 0, b->size * sizeof(data_t));
    } else {
        b->buffer = new data_t[b->size];
        reset(b);
    }
    return b;
}
inline void destructor(Bitmap **const b) {
    if ((*b)->using_cuda) hc_dev_free((*b)->buffer);
    else delete[] (*b)->buffer;
    delete *b;
    *b = nullptr;
}
// Host proxy of a device buffer (src/bitmap.cuh:122-160).
inline Bitmap *cu_cpu_constructor(const std::size_t num_elements) { return constructor(num_elements, true); }
inline void cu_cpu_destructor(Bitmap **const b) { destructor(b); }
inline void cu_cpu_reset(Bitmap *const b) { hc_dev_memset(b->buffer, 0, b->size * sizeof(data_t)); }
inline void cu_cpu_set_bit(Bitmap *const b, const std::size_t idx) {
    data_t w = 0;
    hc_memcpy(&w, b->buffer + data_offset(idx), sizeof(w));
    w |= static_cast<data_t>(1) << bit_offset(idx);
    hc_memcpy(b->buffer + data_offset(idx), &w, sizeof(w));
}
// The struct itself in device memory (src/bitmap.cuh:165-183).
inline Bitmap *cu_constructor(const Bitmap *const b) {
    Bitmap *d = nullptr;
    hc_compat_dev_alloc((void **)&d, sizeof(Bitmap));
    hc_memcpy(d, b, sizeof(Bitmap));
    return d;
}
inline void cu_destructor(Bitmap **const d) {
    hc_dev_free(*d);
    *d = nullptr;
}
}  // namespace Bitmap

// ---------------------------------------------------------------- kernels
// Epoch-kernel types with the reference's signatures
// (src/kernels/kernel_types.cuh:36-63).
typedef void (*sssp_gpu_epoch_func)(const offset_t *, const wnode_t *, const nid_t, const nid_t, weight_t *, nid_t *);
typedef void (*pr_gpu_epoch_func)(const offset_t *, const wnode_t *, const nid_t, const nid_t, weight_t *, nid_t *,
                                  int, offset_t *);
typedef void (*bfs_gpu_epoch_func)(const offset_t *const, const nid_t *const, nid_t *const, const nid_t,
                                   const nid_t, const Bitmap::Bitmap *const, Bitmap::Bitmap *const, nid_t *const);

// The reference's kernel names are functions of those types.  A driver given
// one runs this library's epoch of that granularity (hc_epoch_*), in the
// reference's host loop; the *_auto names run this engine's device-driven
// paths.  Called directly (device pointers, Bitmap structs in host or device
// memory), a name runs one epoch with the drivers' default launch shape.
// Any other function of the same type is taken to be the caller's own
// __global__ epoch kernel: under nvcc the drivers launch it with <<<...>>>
// exactly as the reference's drivers do; elsewhere it is refused.
namespace hc_compat {
constexpr int kDefaultBlocks = 64, kDefaultThreads = 1024;
inline Bitmap::Bitmap read_bitmap(const Bitmap::Bitmap *b) {
    Bitmap::Bitmap h{};
    check(hc_memcpy(&h, b, sizeof(h)), "hc_memcpy");
    return h;
}
inline void bfs_epoch(hc_variant v, int sync_iters, const offset_t *index, const nid_t *nbr, nid_t *parents,
                      nid_t start, nid_t end, const Bitmap::Bitmap *f, Bitmap::Bitmap *nf, nid_t *count) {
    const Bitmap::Bitmap hf = read_bitmap(f), hnf = read_bitmap(nf);
    if (sync_iters > 0)
        check(hc_epoch_bfs_sync_pull(index, nbr, parents, start, end, (const uint32_t *)hf.buffer,
                                     (uint32_t *)hnf.buffer, count, sync_iters, kDefaultBlocks, kDefaultThreads,
                                     nullptr), "hc_epoch_bfs_sync_pull");
    else
        check(hc_epoch_bfs_pull(index, nbr, parents, start, end, (const uint32_t *)hf.buffer, (uint32_t *)hnf.buffer,
                                count, v, kDefaultBlocks, kDefaultThreads, nullptr), "hc_epoch_bfs_pull");
}
}  // namespace hc_compat

inline void epoch_sssp_pull_gpu_one_to_one(const offset_t *i, const wnode_t *n, const nid_t s, const nid_t e,
                                           weight_t *d, nid_t *u) {
    hc_compat::check(hc_epoch_sssp_pull(i, n, s, e, d, u, HC_VARIANT_THREAD, 64, 1024, nullptr), "hc_epoch_sssp_pull");
}
inline void epoch_sssp_pull_gpu_warp_red(const offset_t *i, const wnode_t *n, const nid_t s, const nid_t e,
                                         weight_t *d, nid_t *u) {
    hc_compat::check(hc_epoch_sssp_pull(i, n, s, e, d, u, HC_VARIANT_WARP, 64, 1024, nullptr), "hc_epoch_sssp_pull");
}
inline void epoch_sssp_pull_gpu_block_red(const offset_t *i, const wnode_t *n, const nid_t s, const nid_t e,
                                          weight_t *d, nid_t *u) {
    hc_compat::check(hc_epoch_sssp_pull(i, n, s, e, d, u, HC_VARIANT_BLOCK, 64, 256, nullptr), "hc_epoch_sssp_pull");
}
inline void epoch_sssp_auto(const offset_t *i, const wnode_t *n, const nid_t s, const nid_t e, weight_t *d,
                            nid_t *u) {
    epoch_sssp_pull_gpu_warp_red(i, n, s, e, d, u);  // as an epoch: the warp variant
}
inline void epoch_pr_pull_gpu_one_to_one(const offset_t *i, const wnode_t *n, const nid_t s, const nid_t e,
                                         weight_t *x, nid_t *u, int nn, offset_t *deg) {
    hc_compat::check(hc_epoch_pr_pull(i, n, s, e, x, u, nn, deg, HC_VARIANT_THREAD, 64, 1024, nullptr),
                     "hc_epoch_pr_pull");
}
inline void epoch_pr_pull_gpu_warp_red(const offset_t *i, const wnode_t *n, const nid_t s, const nid_t e,
                                       weight_t *x, nid_t *u, int nn, offset_t *deg) {
    hc_compat::check(hc_epoch_pr_pull(i, n, s, e, x, u, nn, deg, HC_VARIANT_WARP, 64, 1024, nullptr),
                     "hc_epoch_pr_pull");
}
inline void epoch_pr_pull_gpu_block_red(const offset_t *i, const wnode_t *n, const nid_t s, const nid_t e,
                                        weight_t *x, nid_t *u, int nn, offset_t *deg) {
    hc_compat::check(hc_epoch_pr_pull(i, n, s, e, x, u, nn, deg, HC_VARIANT_BLOCK, 64, 256, nullptr),
                     "hc_epoch_pr_pull");
}
inline void epoch_pr_auto(const offset_t *i, const wnode_t *n, const nid_t s, const nid_t e, weight_t *x, nid_t *u,
                          int nn, offset_t *deg) {
    epoch_pr_pull_gpu_one_to_one(i, n, s, e, x, u, nn, deg);
}
inline void epoch_bfs_pull_gpu_one_to_one(const offset_t *const i, const nid_t *const n, nid_t *const p,
                                          const nid_t s, const nid_t e, const Bitmap::Bitmap *const f,
                                          Bitmap::Bitmap *const nf, nid_t *const c) {
    hc_compat::bfs_epoch(HC_VARIANT_THREAD, 0, i, n, p, s, e, f, nf, c);
}
inline void epoch_bfs_pull_gpu_warp(const offset_t *const i, const nid_t *const n, nid_t *const p, const nid_t s,
                                    const nid_t e, const Bitmap::Bitmap *const f, Bitmap::Bitmap *const nf,
                                    nid_t *const c) {
    hc_compat::bfs_epoch(HC_VARIANT_WARP, 0, i, n, p, s, e, f, nf, c);
}
// epoch_bfs_sync_pull_gpu_warp<sync_iters> (src/kernels/gpu/bfs.cuh:234-288):
// callers name it with or without the template argument, as the reference's do
// (tests/bfs/bfs_verify.cu, profile/bfs/benchmark_bfs.cu:242-260).
template <offset_t sync_iters = 1>
inline void epoch_bfs_sync_pull_gpu_warp(const offset_t *const i, const nid_t *const n, nid_t *const p,
                                         const nid_t s, const nid_t e, const Bitmap::Bitmap *const f,
                                         Bitmap::Bitmap *const nf, nid_t *const c) {
    static_assert(sync_iters >= 1, "sync_iters must be at least 1");
    hc_compat::bfs_epoch(HC_VARIANT_WARP, (int)sync_iters, i, n, p, s, e, f, nf, c);
}
inline void epoch_bfs_auto(const offset_t *const i, const nid_t *const n, nid_t *const p, const nid_t s,
                           const nid_t e, const Bitmap::Bitmap *const f, Bitmap::Bitmap *const nf, nid_t *const c) {
    hc_compat::bfs_epoch(HC_VARIANT_THREAD, 0, i, n, p, s, e, f, nf, c);
}

namespace hc_compat {
// What a driver does with a kernel name: this library's epoch of a
// granularity, the engine path, or (not found) the caller's own kernel.
struct KernelInfo {
    hc_variant variant;
    bool engine;
    int sync_iters;
    const char *name;
};
constexpr int kMaxSyncIters = 8;
template <int K>
inline void add_sync(std::vector<std::pair<bfs_gpu_epoch_func, KernelInfo>> &v) {
    if constexpr (K >= 1) {
        add_sync<K - 1>(v);
        static const std::string name = "bfs_gpu_sync_warp_" + std::to_string(K);
        v.push_back({&epoch_bfs_sync_pull_gpu_warp<K>, {HC_VARIANT_WARP, false, K, name.c_str()}});
    }
}
inline const KernelInfo *lookup(bfs_gpu_epoch_func f) {
    static const std::vector<std::pair<bfs_gpu_epoch_func, KernelInfo>> table = [] {
        std::vector<std::pair<bfs_gpu_epoch_func, KernelInfo>> v = {
            {&epoch_bfs_pull_gpu_one_to_one, {HC_VARIANT_THREAD, false, 0, "bfs_gpu_onetoone"}},
            {&epoch_bfs_pull_gpu_warp, {HC_VARIANT_WARP, false, 0, "bfs_gpu_warp"}},
            {&epoch_bfs_auto, {HC_VARIANT_AUTO, true, 0, "bfs_gpu_auto"}}};
        add_sync<kMaxSyncIters>(v);
        return v;
    }();
    for (auto &e : table)
        if (e.first == f) return &e.second;
    return nullptr;
}
inline const KernelInfo *lookup(sssp_gpu_epoch_func f) {
    static const std::pair<sssp_gpu_epoch_func, KernelInfo> table[] = {
        {&epoch_sssp_pull_gpu_one_to_one, {HC_VARIANT_THREAD, false, 0, "sssp_gpu_onetoone"}},
        {&epoch_sssp_pull_gpu_warp_red, {HC_VARIANT_WARP, false, 0, "sssp_gpu_warp_red"}},
        {&epoch_sssp_pull_gpu_block_red, {HC_VARIANT_BLOCK, false, 0, "sssp_gpu_block_red"}},
        {&epoch_sssp_auto, {HC_VARIANT_AUTO, true, 0, "sssp_gpu_auto"}}};
    for (auto &e : table)
        if (e.first == f) return &e.second;
    return nullptr;
}
inline const KernelInfo *lookup(pr_gpu_epoch_func f) {
    static const std::pair<pr_gpu_epoch_func, KernelInfo> table[] = {
        {&epoch_pr_pull_gpu_one_to_one, {HC_VARIANT_THREAD, false, 0, "pr_gpu_onetoone"}},
        {&epoch_pr_pull_gpu_warp_red, {HC_VARIANT_WARP, false, 0, "pr_gpu_warp_red"}},
        {&epoch_pr_pull_gpu_block_red, {HC_VARIANT_BLOCK, false, 0, "pr_gpu_block_red"}},
        {&epoch_pr_auto, {HC_VARIANT_AUTO, true, 0, "pr_gpu_auto"}}};
    for (auto &e : table)
        if (e.first == f) return &e.second;
    return nullptr;
}
// A caller's own kernel (not one of the names above): launched as the
// reference's drivers launch theirs, when compiled by nvcc.
[[noreturn]] inline void no_user_kernels(const char *who) {
    std::cerr << "[" << who << "] the epoch kernel is not one of this library's names; a kernel of your own "
              << "needs this header compiled by nvcc" << std::endl;
    std::exit(EXIT_FAILURE);
}
}  // namespace hc_compat

enum class BFSGPU { one_to_one, warp, automatic, undefined };
enum class SSSPGPU { one_to_one, warp_red, block_red, automatic, undefined };
enum class PRGPU { one_to_one, warp_red, block_red, automatic, undefined };

inline std::vector<BFSGPU> get_kernels(BFSGPU) { return {BFSGPU::one_to_one, BFSGPU::warp, BFSGPU::automatic}; }
inline std::vector<SSSPGPU> get_kernels(SSSPGPU) {
    return {SSSPGPU::one_to_one, SSSPGPU::warp_red, SSSPGPU::block_red, SSSPGPU::automatic};
}
inline std::vector<PRGPU> get_kernels(PRGPU) {
    return {PRGPU::one_to_one, PRGPU::warp_red, PRGPU::block_red, PRGPU::automatic};
}

inline bfs_gpu_epoch_func get_kernel(BFSGPU k) {
    switch (k) {
        case BFSGPU::one_to_one: return epoch_bfs_pull_gpu_one_to_one;
        case BFSGPU::warp: return epoch_bfs_pull_gpu_warp;
        case BFSGPU::automatic: return epoch_bfs_auto;
        default: return nullptr;
    }
}
inline sssp_gpu_epoch_func get_kernel(SSSPGPU k) {
    switch (k) {
        case SSSPGPU::one_to_one: return epoch_sssp_pull_gpu_one_to_one;
        case SSSPGPU::warp_red: return epoch_sssp_pull_gpu_warp_red;
        case SSSPGPU::block_red: return epoch_sssp_pull_gpu_block_red;
        case SSSPGPU::automatic: return epoch_sssp_auto;
        default: return nullptr;
    }
}
inline pr_gpu_epoch_func get_kernel(PRGPU k) {
    switch (k) {
        case PRGPU::one_to_one: return epoch_pr_pull_gpu_one_to_one;
        case PRGPU::warp_red: return epoch_pr_pull_gpu_warp_red;
        case PRGPU::block_red: return epoch_pr_pull_gpu_block_red;
        case PRGPU::automatic: return epoch_pr_auto;
        default: return nullptr;
    }
}
template <class E>
inline std::string to_repr(E k) {
    auto f = get_kernel(k);
    const hc_compat::KernelInfo *i = f ? hc_compat::lookup(f) : nullptr;
    return i ? i->name : "";
}
template <class E>
inline std::string to_string(E k) {
    const std::string r = to_repr(k);
    return r.empty() ? "undefined GPU kernel" : "GPU " + r;
}

// ---------------------------------------------------------------- drivers

namespace hc_compat {
struct DevArray {
    void *p = nullptr;
    DevArray(size_t bytes) { check(hc_dev_malloc(&p, bytes, 0), "hc_dev_malloc"); }
    ~DevArray() { hc_dev_free(p); }
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};
inline double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace hc_compat

// bfs_gpu (src/kernels/gpu/bfs.cuh:21-95): parents from source_id.
inline double bfs_gpu(const CSRUWGraph &g, const nid_t source_id, nid_t **const ret_parents,
                      bfs_gpu_epoch_func epoch_kernel, int block_count = 64, int thread_count = 1024) {
    using namespace hc_compat;
    if (!epoch_kernel) check(HC_ERR_INVALID_ARG, "bfs_gpu: null epoch kernel");
    const KernelInfo *ki = lookup(epoch_kernel);
#ifndef __CUDACC__
    if (!ki) no_user_kernels("bfs_gpu");
#endif
    nid_t *parents = new nid_t[g.num_nodes];
    double ms = 0;
    if (ki && ki->engine) {
        hc_graph *hg = nullptr;
        check(hc_graph_create(g.index, g.neighbors, nullptr, HC_W_NONE, g.num_nodes, g.num_edges, 0, &hg),
              "hc_graph_create");
        hc_bfs_stats st{};
        check(hc_bfs(hg, &source_id, 1, nullptr, parents, nullptr, &st), "hc_bfs");
        ms = st.ms;
        hc_graph_destroy(hg);
    } else {
        const size_t words = ((size_t)g.num_nodes + 31) / 32;
        DevArray idx(8 * ((size_t)g.num_nodes + 1)), nbr(4 * (size_t)g.num_edges + 4),
            par(4 * (size_t)g.num_nodes), f0(4 * words), f1(4 * words), cnt(4);
        check(hc_memcpy(idx.p, g.index, 8 * ((size_t)g.num_nodes + 1)), "hc_memcpy");
        check(hc_memcpy(nbr.p, g.neighbors, 4 * (size_t)g.num_edges), "hc_memcpy");
        check(hc_csr_check(idx.as<int64_t>(), nbr.p, 0, g.num_nodes, g.num_edges, nullptr), "hc_csr_check");
        for (nid_t i = 0; i < g.num_nodes; i++) parents[i] = INVALID_NODE;
        parents[source_id] = source_id;
        check(hc_memcpy(par.p, parents, 4 * (size_t)g.num_nodes), "hc_memcpy");
        check(hc_dev_memset(f0.p, 0, 4 * words), "hc_dev_memset");
        uint32_t bit = 1u << (source_id & 31);
        check(hc_memcpy(f0.as<uint32_t>() + (source_id >> 5), &bit, 4), "hc_memcpy");
        // Device Bitmap structs over the two frontier buffers, as the
        // reference's driver builds them (src/bitmap.cuh:165-183).
        Bitmap::Bitmap hb[2] = {{f0.as<int>(), true, words}, {f1.as<int>(), true, words}};
        Bitmap::Bitmap *cb[2] = {Bitmap::cu_constructor(&hb[0]), Bitmap::cu_constructor(&hb[1])};
        int cur = 0;
        auto t0 = std::chrono::steady_clock::now();
        nid_t found = 0;
        do {
            check(hc_dev_memset(cnt.p, 0, 4), "hc_dev_memset");
            check(hc_dev_memset(hb[1 - cur].buffer, 0, 4 * words), "hc_dev_memset");
            if (!ki) {
#ifdef __CUDACC__
                (*epoch_kernel)<<<block_count, thread_count>>>(idx.as<offset_t>(), nbr.as<nid_t>(), par.as<nid_t>(), 0,
                                                              g.num_nodes, cb[cur], cb[1 - cur], cnt.as<nid_t>());
                check(cudaGetLastError() == cudaSuccess ? HC_OK : HC_ERR_CUDA, "bfs_gpu: epoch launch");
#endif
            } else if (ki->sync_iters > 0) {
                check(hc_epoch_bfs_sync_pull(idx.as<int64_t>(), nbr.as<int32_t>(), par.as<int32_t>(), 0, g.num_nodes,
                                             (const uint32_t *)hb[cur].buffer, (uint32_t *)hb[1 - cur].buffer,
                                             cnt.as<int32_t>(), ki->sync_iters, block_count, thread_count, nullptr),
                      "hc_epoch_bfs_sync_pull");
            } else {
                check(hc_epoch_bfs_pull(idx.as<int64_t>(), nbr.as<int32_t>(), par.as<int32_t>(), 0, g.num_nodes,
                                        (const uint32_t *)hb[cur].buffer, (uint32_t *)hb[1 - cur].buffer,
                                        cnt.as<int32_t>(), ki->variant, block_count, thread_count, nullptr),
                      "hc_epoch_bfs_pull");
            }
            check(hc_memcpy(&found, cnt.p, 4), "hc_memcpy");
            cur = 1 - cur;
        } while (found != 0);
        ms = ms_since(t0);
        Bitmap::cu_destructor(&cb[0]);
        Bitmap::cu_destructor(&cb[1]);
        check(hc_memcpy(parents, par.p, 4 * (size_t)g.num_nodes), "hc_memcpy");
    }
    *ret_parents = parents;
    return ms;
}

// sssp_pull_gpu (src/kernels/gpu/sssp.cuh:42-100): distances from init_dist.
inline double sssp_pull_gpu(const CSRWGraph &g, sssp_gpu_epoch_func epoch_kernel, const weight_t *init_dist,
                            weight_t **const ret_dist, int block_count = 64, int thread_count = 1024) {
    using namespace hc_compat;
    if (!epoch_kernel) check(HC_ERR_INVALID_ARG, "sssp_pull_gpu: null epoch kernel");
    const KernelInfo *ki = lookup(epoch_kernel);
#ifndef __CUDACC__
    if (!ki) no_user_kernels("sssp_pull_gpu");
#endif
    weight_t *dist = new weight_t[g.num_nodes];
    double ms = 0;
    // The engine path needs one source (a single 0, the rest inf) and
    // integer weights; anything else runs the epoch loop.
    nid_t src = -1;
    bool single = ki && ki->engine;
    for (nid_t i = 0; single && i < g.num_nodes; i++) {
        if (init_dist[i] == 0.0f && src < 0) src = i;
        else if (!std::isinf(init_dist[i])) single = false;
    }
    std::vector<int32_t> w;
    if (single && src >= 0) {
        w.resize((size_t)g.num_edges);
        for (offset_t i = 0; i < g.num_edges && single; i++) {
            float x = g.neighbors[i].w;
            single = x >= 0.f && x < 2147483520.f && std::floor(x) == x;
            w[i] = (int32_t)x;
        }
    }
    if (single && src >= 0) {
        std::vector<int32_t> nbr((size_t)g.num_edges);
        for (offset_t i = 0; i < g.num_edges; i++) nbr[i] = g.neighbors[i].v;
        hc_graph *hg = nullptr;
        check(hc_graph_create(g.index, nbr.data(), w.data(), HC_W_I32, g.num_nodes, g.num_edges, 0, &hg),
              "hc_graph_create");
        std::vector<int32_t> d((size_t)g.num_nodes);
        hc_sssp_stats st{};
        check(hc_sssp(hg, &src, 1, d.data(), nullptr, nullptr, &st), "hc_sssp");
        ms = st.ms;
        hc_graph_destroy(hg);
        for (nid_t i = 0; i < g.num_nodes; i++) dist[i] = d[i] == 0x7fffffff ? INF_WEIGHT : (weight_t)d[i];
    } else {
        DevArray idx(8 * ((size_t)g.num_nodes + 1)), nb(8 * (size_t)g.num_edges + 8), dd(4 * (size_t)g.num_nodes),
            cnt(4);
        check(hc_memcpy(idx.p, g.index, 8 * ((size_t)g.num_nodes + 1)), "hc_memcpy");
        check(hc_memcpy(nb.p, g.neighbors, 8 * (size_t)g.num_edges), "hc_memcpy");
        check(hc_memcpy(dd.p, init_dist, 4 * (size_t)g.num_nodes), "hc_memcpy");
        check(hc_csr_check(idx.as<int64_t>(), nb.p, 1, g.num_nodes, g.num_edges, nullptr), "hc_csr_check");
        auto t0 = std::chrono::steady_clock::now();
        nid_t updated = 1;
        while (updated != 0) {
            check(hc_dev_memset(cnt.p, 0, 4), "hc_dev_memset");
            if (!ki) {
#ifdef __CUDACC__
                (*epoch_kernel)<<<block_count, thread_count>>>(idx.as<offset_t>(), nb.as<wnode_t>(), 0, g.num_nodes,
                                                              dd.as<weight_t>(), cnt.as<nid_t>());
                check(cudaGetLastError() == cudaSuccess ? HC_OK : HC_ERR_CUDA, "sssp_pull_gpu: epoch launch");
#endif
            } else {
                check(hc_epoch_sssp_pull(idx.as<int64_t>(), nb.p, 0, g.num_nodes, dd.as<float>(), cnt.as<int32_t>(),
                                         ki->variant == HC_VARIANT_AUTO ? HC_VARIANT_WARP : ki->variant, block_count,
                                         thread_count, nullptr),
                      "hc_epoch_sssp_pull");
            }
            check(hc_memcpy(&updated, cnt.p, 4), "hc_memcpy");
        }
        ms = ms_since(t0);
        check(hc_memcpy(dist, dd.p, 4 * (size_t)g.num_nodes), "hc_memcpy");
    }
    *ret_dist = dist;
    return ms;
}

// pr_pull_gpu (src/kernels/gpu/pr.cuh:42-118): at most 201 epochs, stops
// when no vertex moves by more than 5e-8.  With epoch_pr_auto the sweeps run
// in the reference's single-thread vertex order (hc_pr_pull_ordered), so the
// scores equal pr_pull_cpu's on one thread bit for bit; the named epoch
// kernels run the reference's own host loop, whose order (and so its stopping
// point) varies with the thread schedule, as the reference's does.
inline double pr_pull_gpu(const CSRWGraph &g, pr_gpu_epoch_func epoch_kernel, weight_t *init_score,
                          weight_t **const ret_score, int block_count = 64, int thread_count = 1024) {
    using namespace hc_compat;
    if (!epoch_kernel) check(HC_ERR_INVALID_ARG, "pr_pull_gpu: null epoch kernel");
    const KernelInfo *ki = lookup(epoch_kernel);
#ifndef __CUDACC__
    if (!ki) no_user_kernels("pr_pull_gpu");
#endif
    weight_t *score = new weight_t[g.num_nodes];
    double ms = 0;
    if (ki && ki->engine) {
        std::vector<int32_t> nbr((size_t)g.num_edges);
        for (offset_t i = 0; i < g.num_edges; i++) nbr[i] = g.neighbors[i].v;
        hc_graph *hg = nullptr;
        check(hc_graph_create(g.index, nbr.data(), nullptr, HC_W_NONE, g.num_nodes, g.num_edges, 0, &hg),
              "hc_graph_create");
        hc_pr_opts o{};
        o.damping = 0.85f;
        o.eps_vertex = 5e-8f;
        o.max_iters = 201;
        hc_pr_stats st{};
        check(hc_pr_pull_ordered(hg, init_score, score, &o, &st), "hc_pr_pull_ordered");
        ms = st.ms;
        hc_graph_destroy(hg);
    } else {
        std::vector<offset_t> deg((size_t)g.num_nodes);
        for (nid_t i = 0; i < g.num_nodes; i++) deg[i] = g.get_degree(i);
        DevArray idx(8 * ((size_t)g.num_nodes + 1)), nb(8 * (size_t)g.num_edges + 8), sc(4 * (size_t)g.num_nodes),
            dg(8 * (size_t)g.num_nodes), cnt(4);
        check(hc_memcpy(idx.p, g.index, 8 * ((size_t)g.num_nodes + 1)), "hc_memcpy");
        check(hc_memcpy(nb.p, g.neighbors, 8 * (size_t)g.num_edges), "hc_memcpy");
        check(hc_memcpy(sc.p, init_score, 4 * (size_t)g.num_nodes), "hc_memcpy");
        check(hc_memcpy(dg.p, deg.data(), 8 * (size_t)g.num_nodes), "hc_memcpy");
        check(hc_csr_check(idx.as<int64_t>(), nb.p, 1, g.num_nodes, g.num_edges, nullptr), "hc_csr_check");
        auto t0 = std::chrono::steady_clock::now();
        nid_t updated = 1;
        for (int it = 0; updated != 0 && it <= 200; it++) {
            check(hc_dev_memset(cnt.p, 0, 4), "hc_dev_memset");
            if (!ki) {
#ifdef __CUDACC__
                (*epoch_kernel)<<<block_count, thread_count>>>(idx.as<offset_t>(), nb.as<wnode_t>(), 0, g.num_nodes,
                                                              sc.as<weight_t>(), cnt.as<nid_t>(), g.num_nodes,
                                                              dg.as<offset_t>());
                check(cudaGetLastError() == cudaSuccess ? HC_OK : HC_ERR_CUDA, "pr_pull_gpu: epoch launch");
#endif
            } else {
                check(hc_epoch_pr_pull(idx.as<int64_t>(), nb.p, 0, g.num_nodes, sc.as<float>(), cnt.as<int32_t>(),
                                       g.num_nodes, dg.as<int64_t>(), ki->variant, block_count, thread_count, nullptr),
                      "hc_epoch_pr_pull");
            }
            check(hc_memcpy(&updated, cnt.p, 4), "hc_memcpy");
        }
        ms = ms_since(t0);
        check(hc_memcpy(score, sc.p, 4 * (size_t)g.num_nodes), "hc_memcpy");
    }
    *ret_score = score;
    return ms;
}

// The reference's heterogeneous drivers (src/kernels/heterogeneous/*.cuh,
// generated code that splits vertex segments over CPUs and GPUs and exchanges
// them peer to peer): here the split collapses to one GPU, and each runs the
// engine path of its algorithm.  enable_all_peer_access* have nothing to do.
inline void enable_all_peer_access() {}
inline void enable_all_peer_access_pr() {}
inline double bfs_do_heterogeneous(const CSRUWGraph &g, const nid_t source_id, nid_t **const ret_parents) {
    return bfs_gpu(g, source_id, ret_parents, epoch_bfs_auto);
}
inline double sssp_pull_heterogeneous(const CSRWGraph &g, const weight_t *init_dist, weight_t **const ret_dist) {
    return sssp_pull_gpu(g, epoch_sssp_auto, init_dist, ret_dist);
}
inline double pr_pull_heterogeneous(const CSRWGraph &g, const weight_t *init_score, weight_t **const ret_score) {
    return pr_pull_gpu(g, epoch_pr_auto, const_cast<weight_t *>(init_score), ret_score);
}

template <class E, class = typename std::enable_if<std::is_enum<E>::value>::type>
inline std::ostream &operator<<(std::ostream &os, E k) {
    return os << to_string(k);
}
