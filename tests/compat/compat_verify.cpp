// Drives the reference-shaped C++ API (include/hc_compat.hpp) the way the
// reference's tests drive theirs (tests/bfs/bfs_verify.cu,
// tests/sssp/sssp_verify.cu, tests/pr/pr_verify.cu): load a graph file, pick
// a source with SourcePicker, run every registered GPU kernel through its
// driver and verify it against a serial computation.  Exit status 0 only if
// every check passes.
//
//   compat_verify graph.sg graph.wsg
#include <cmath>
#include <cstdio>
#include <deque>
#include <functional>
#include <queue>

#include "hc_compat.hpp"

static int failures = 0;

static std::vector<nid_t> serial_depth(const CSRUWGraph &g, nid_t src) {
    std::vector<nid_t> d(g.num_nodes, INVALID_NODE);
    std::deque<nid_t> q{src};
    d[src] = 0;
    while (!q.empty()) {
        nid_t u = q.front();
        q.pop_front();
        for (offset_t i = g.index[u]; i < g.index[u + 1]; i++)
            if (d[g.neighbors[i]] == INVALID_NODE) {
                d[g.neighbors[i]] = d[u] + 1;
                q.push_back(g.neighbors[i]);
            }
    }
    return d;
}

static std::vector<weight_t> serial_sssp(const CSRWGraph &g, nid_t src) {
    std::vector<weight_t> d(g.num_nodes, INF_WEIGHT);
    using P = std::pair<weight_t, nid_t>;
    std::priority_queue<P, std::vector<P>, std::greater<P>> pq;
    d[src] = 0;
    pq.push({0.f, src});
    while (!pq.empty()) {
        auto [w, u] = pq.top();
        pq.pop();
        if (w != d[u]) continue;
        for (offset_t i = g.index[u]; i < g.index[u + 1]; i++) {
            weight_t nd = w + g.neighbors[i].w;
            if (nd < d[g.neighbors[i].v]) {
                d[g.neighbors[i].v] = nd;
                pq.push({nd, g.neighbors[i].v});
            }
        }
    }
    return d;
}

// Jacobi power iteration in double to a tight tolerance.
static std::vector<double> serial_pr(const CSRWGraph &g) {
    const nid_t n = g.num_nodes;
    std::vector<double> x(n, 1.0 / n), y(n);
    for (int it = 0; it < 1000; it++) {
        double l1 = 0;
        for (nid_t v = 0; v < n; v++) {
            double s = 0;
            for (offset_t i = g.index[v]; i < g.index[v + 1]; i++) {
                nid_t u = g.neighbors[i].v;
                s += x[u] / (double)g.get_degree(u);
            }
            y[v] = 0.15 / n + 0.85 * s;
            l1 += std::fabs(y[v] - x[v]);
        }
        x.swap(y);
        if (l1 < 1e-13) break;
    }
    return x;
}

static void report(const std::string &name, bool ok, const std::string &detail) {
    std::cout << "Verifying " << name << " kernel ... " << (ok ? "success" : "FAILED") << " " << detail
              << std::endl;
    if (!ok) failures++;
}

int main(int argc, char *argv[]) {
    if (argc != 3) {
        std::cerr << "Usage: " << argv[0] << " [graph.sg] [graph.wsg]" << std::endl;
        return EXIT_FAILURE;
    }
    {
        CSRUWGraph g = load_graph_from_file<CSRUWGraph>(argv[1]);
        SourcePicker<CSRUWGraph> sp(&g);
        nid_t source_id = sp.next_vertex();
        std::vector<nid_t> depth = serial_depth(g, source_id);
        auto check_bfs = [&](const std::string &name, bfs_gpu_epoch_func kernel) {
            nid_t *parents = nullptr;
            bfs_gpu(g, source_id, &parents, kernel);
            nid_t bad = 0;
            for (nid_t u = 0; u < g.num_nodes; u++) {
                if (parents[u] == INVALID_NODE) bad += depth[u] != INVALID_NODE;
                else if (u == source_id) bad += parents[u] != source_id;
                else bad += depth[u] != depth[parents[u]] + 1;
            }
            report(name, bad == 0, std::to_string(bad) + " bad parents");
            delete[] parents;
        };
        for (BFSGPU k : get_kernels(BFSGPU::undefined)) check_bfs(to_string(k), get_kernel(k));
        // The sync-warp kernel as profile/bfs/benchmark_bfs.cu:242-260 names it.
        check_bfs("GPU sync warp (sync_iters = 1)", epoch_bfs_sync_pull_gpu_warp<1>);
        check_bfs("GPU sync warp (sync_iters = 2)", epoch_bfs_sync_pull_gpu_warp<2>);
        check_bfs("GPU sync warp (sync_iters = 3)", epoch_bfs_sync_pull_gpu_warp<3>);
    }
    {
        CSRWGraph g = load_graph_from_file<CSRWGraph>(argv[2]);
        SourcePicker<CSRWGraph> sp(&g);
        nid_t source_id = sp.next_vertex();
        std::vector<weight_t> oracle = serial_sssp(g, source_id);
        std::vector<weight_t> init(g.num_nodes, INF_WEIGHT);
        init[source_id] = 0;
        for (SSSPGPU k : get_kernels(SSSPGPU::undefined)) {
            weight_t *dist = nullptr;
            sssp_pull_gpu(g, get_kernel(k), init.data(), &dist, 64, 256);
            nid_t bad = 0;
            for (nid_t u = 0; u < g.num_nodes; u++) bad += dist[u] != oracle[u];
            report(to_string(k), bad == 0, std::to_string(bad) + " wrong distances");
            delete[] dist;
        }
        std::vector<double> x = serial_pr(g);
        std::vector<weight_t> init_score(g.num_nodes, 1.0f / g.num_nodes);
        for (PRGPU k : get_kernels(PRGPU::undefined)) {
            weight_t *score = nullptr;
            pr_pull_gpu(g, get_kernel(k), init_score.data(), &score, 64, 256);
            double err = 0;
            for (nid_t u = 0; u < g.num_nodes; u++) err = std::max(err, std::fabs(score[u] - x[u]));
            // The reference test accepts |diff| <= 5e-4 (tests/pr/pr_verify.cu:132);
            // this one asks for 1e-5 against the FP64 fixed point.
            report(to_string(k), err <= 1e-5, "max |diff| vs FP64 " + std::to_string(err));
            delete[] score;
        }
    }
    std::cout << (failures ? "FAILED" : "ALL OK") << std::endl;
    return failures ? EXIT_FAILURE : EXIT_SUCCESS;
}
