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

// ---------------------------------------------------------------- kernels

struct hc_epoch_kernel {
    hc_variant variant;
    bool engine;  // true: this library's device-driven path
    const char *name;
    int sync_iters;  // > 0: the sync-warp BFS epoch probing that many chunks per vote
};
using bfs_gpu_epoch_func = const hc_epoch_kernel *;
using sssp_gpu_epoch_func = const hc_epoch_kernel *;
using pr_gpu_epoch_func = const hc_epoch_kernel *;

inline const hc_epoch_kernel hc_k_bfs_one[] = {{HC_VARIANT_THREAD, false, "bfs_gpu_onetoone"}};
inline const hc_epoch_kernel hc_k_bfs_warp[] = {{HC_VARIANT_WARP, false, "bfs_gpu_warp"}};
inline const hc_epoch_kernel hc_k_bfs_auto[] = {{HC_VARIANT_AUTO, true, "bfs_gpu_auto"}};
inline const hc_epoch_kernel hc_k_sssp_one[] = {{HC_VARIANT_THREAD, false, "sssp_gpu_onetoone"}};
inline const hc_epoch_kernel hc_k_sssp_warp[] = {{HC_VARIANT_WARP, false, "sssp_gpu_warp_red"}};
inline const hc_epoch_kernel hc_k_sssp_block[] = {{HC_VARIANT_BLOCK, false, "sssp_gpu_block_red"}};
inline const hc_epoch_kernel hc_k_sssp_auto[] = {{HC_VARIANT_AUTO, true, "sssp_gpu_auto"}};
inline const hc_epoch_kernel hc_k_pr_one[] = {{HC_VARIANT_THREAD, false, "pr_gpu_onetoone"}};
inline const hc_epoch_kernel hc_k_pr_warp[] = {{HC_VARIANT_WARP, false, "pr_gpu_warp_red"}};
inline const hc_epoch_kernel hc_k_pr_block[] = {{HC_VARIANT_BLOCK, false, "pr_gpu_block_red"}};
inline const hc_epoch_kernel hc_k_pr_auto[] = {{HC_VARIANT_AUTO, true, "pr_gpu_auto"}};

// Reference kernel names (src/kernels/gpu/*.cuh).
inline const bfs_gpu_epoch_func epoch_bfs_pull_gpu_one_to_one = hc_k_bfs_one;
inline const bfs_gpu_epoch_func epoch_bfs_pull_gpu_warp = hc_k_bfs_warp;
// epoch_bfs_sync_pull_gpu_warp<sync_iters> (src/kernels/gpu/bfs.cuh:234-288),
// spelled as the reference's callers spell it (`epoch_bfs_sync_pull_gpu_warp<2>`).
template <offset_t sync_iters = 1>
inline const hc_epoch_kernel hc_k_bfs_sync[] = {{HC_VARIANT_WARP, false, "bfs_gpu_sync_warp", (int)sync_iters}};
template <offset_t sync_iters = 1>
inline const bfs_gpu_epoch_func epoch_bfs_sync_pull_gpu_warp = hc_k_bfs_sync<sync_iters>;
inline const bfs_gpu_epoch_func epoch_bfs_auto = hc_k_bfs_auto;
inline const sssp_gpu_epoch_func epoch_sssp_pull_gpu_one_to_one = hc_k_sssp_one;
inline const sssp_gpu_epoch_func epoch_sssp_pull_gpu_warp_red = hc_k_sssp_warp;
inline const sssp_gpu_epoch_func epoch_sssp_pull_gpu_block_red = hc_k_sssp_block;
inline const sssp_gpu_epoch_func epoch_sssp_auto = hc_k_sssp_auto;
inline const pr_gpu_epoch_func epoch_pr_pull_gpu_one_to_one = hc_k_pr_one;
inline const pr_gpu_epoch_func epoch_pr_pull_gpu_warp_red = hc_k_pr_warp;
inline const pr_gpu_epoch_func epoch_pr_pull_gpu_block_red = hc_k_pr_block;
inline const pr_gpu_epoch_func epoch_pr_auto = hc_k_pr_auto;

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
    return f ? f->name : "";
}
template <class E>
inline std::string to_string(E k) {
    auto f = get_kernel(k);
    return f ? std::string("GPU ") + f->name : "undefined GPU kernel";
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
    nid_t *parents = new nid_t[g.num_nodes];
    double ms = 0;
    if (epoch_kernel->engine) {
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
        uint32_t *cur = f0.as<uint32_t>(), *next = f1.as<uint32_t>();
        auto t0 = std::chrono::steady_clock::now();
        nid_t found = 0;
        do {
            check(hc_dev_memset(cnt.p, 0, 4), "hc_dev_memset");
            check(hc_dev_memset(next, 0, 4 * words), "hc_dev_memset");
            if (epoch_kernel->sync_iters > 0)
                check(hc_epoch_bfs_sync_pull(idx.as<int64_t>(), nbr.as<int32_t>(), par.as<int32_t>(), 0, g.num_nodes,
                                             cur, next, cnt.as<int32_t>(), epoch_kernel->sync_iters, block_count,
                                             thread_count, nullptr),
                      "hc_epoch_bfs_sync_pull");
            else
                check(hc_epoch_bfs_pull(idx.as<int64_t>(), nbr.as<int32_t>(), par.as<int32_t>(), 0, g.num_nodes, cur,
                                        next, cnt.as<int32_t>(), epoch_kernel->variant, block_count, thread_count,
                                        nullptr),
                      "hc_epoch_bfs_pull");
            check(hc_memcpy(&found, cnt.p, 4), "hc_memcpy");
            std::swap(cur, next);
        } while (found != 0);
        ms = ms_since(t0);
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
    weight_t *dist = new weight_t[g.num_nodes];
    double ms = 0;
    // The engine path needs one source (a single 0, the rest inf) and
    // integer weights; anything else runs the epoch loop.
    nid_t src = -1;
    bool single = epoch_kernel->engine;
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
            check(hc_epoch_sssp_pull(idx.as<int64_t>(), nb.p, 0, g.num_nodes, dd.as<float>(), cnt.as<int32_t>(),
                                     epoch_kernel->variant == HC_VARIANT_AUTO ? HC_VARIANT_WARP : epoch_kernel->variant,
                                     block_count, thread_count, nullptr),
                  "hc_epoch_sssp_pull");
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
    weight_t *score = new weight_t[g.num_nodes];
    double ms = 0;
    if (epoch_kernel->engine) {
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
            check(hc_epoch_pr_pull(idx.as<int64_t>(), nb.p, 0, g.num_nodes, sc.as<float>(), cnt.as<int32_t>(),
                                   g.num_nodes, dg.as<int64_t>(), epoch_kernel->variant, block_count, thread_count,
                                   nullptr),
                  "hc_epoch_pr_pull");
            check(hc_memcpy(&updated, cnt.p, 4), "hc_memcpy");
        }
        ms = ms_since(t0);
        check(hc_memcpy(score, sc.p, 4 * (size_t)g.num_nodes), "hc_memcpy");
    }
    *ret_score = score;
    return ms;
}

template <class E, class = typename std::enable_if<std::is_enum<E>::value>::type>
inline std::ostream &operator<<(std::ostream &os, E k) {
    return os << to_string(k);
}
