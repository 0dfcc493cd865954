/*
 * ref_driver.cu -- TEST INFRASTRUCTURE ONLY.  Runs the reference's own CPU
 * implementation (chrisliu/hetero-compute, compiled unchanged from its source
 * tree by oracle/Makefile) on a .sg / .wsg graph file, for two purposes:
 *   - pinning the oracle: tests/golden/make_golden.py stores its outputs;
 *   - the timed CPU baseline of bench.py (kind "reference").
 *
 * Usage: ref_driver <bfs|sssp|sssp_dijkstra|pr> <graph> <num_sources> <out.bin|->
 *                   [repeats [warmup]]
 * Sources come from the reference's SourcePicker (src/graph.cuh:106-141).
 * The graph is loaded once; `warmup` untimed runs (from the first source) come
 * first, then the source sequence runs `repeats` times (outputs of the first
 * pass only are written).  Prints one JSON line: sources, per-run
 * milliseconds as returned by the reference drivers (epoch loop only; repeats
 * x num_sources entries, repeats for pr), OpenMP threads used.
 *
 * Reference code called:
 *   bfs_do_cpu<15,18>            src/kernels/cpu/bfs.cuh:48-114
 *   sssp_pull_cpu                src/kernels/cpu/sssp.cuh:33-65 (+ epoch :155-182)
 *   sssp_dijkstras_cpu_serial    src/kernels/cpu/sssp.cuh:74-109
 *   pr_pull_cpu                  src/kernels/cpu/pr.cuh:33-65 (+ epoch :157-187)
 */
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "src/graph.cuh"
#include "src/kernels/cpu/bfs.cuh"
#include "src/kernels/cpu/pr.cuh"
#include "src/kernels/cpu/sssp.cuh"

static void write_out(FILE *f, const void *p, size_t bytes) {
    if (f && bytes && fwrite(p, 1, bytes, f) != bytes) {
        std::fprintf(stderr, "write failed\n");
        std::exit(2);
    }
}

int main(int argc, char **argv) {
    if (argc < 5 || argc > 7) {
        std::fprintf(stderr, "usage: %s <bfs|sssp|sssp_dijkstra|pr> <graph> <num_sources> <out.bin|-> [repeats "
                     "[warmup]]\n", argv[0]);
        return 1;
    }
    const std::string algo = argv[1];
    char *path = argv[2];
    const int nsrc = std::atoi(argv[3]);
    const int repeats = argc > 5 ? std::max(1, std::atoi(argv[5])) : 1;
    const int warmup = argc > 6 ? std::max(0, std::atoi(argv[6])) : 0;
    FILE *out = std::strcmp(argv[4], "-") ? std::fopen(argv[4], "wb") : nullptr;
    if (std::strcmp(argv[4], "-") && !out) {
        std::fprintf(stderr, "cannot open %s\n", argv[4]);
        return 1;
    }
    std::vector<int> sources;
    std::vector<double> ms;
    long long n = 0, m = 0;
    int iters = 0;

    if (algo == "bfs") {
        CSRUWGraph g = load_graph_from_file<CSRUWGraph>(path);
        n = g.num_nodes;
        m = g.num_edges;
        for (int r = -warmup; r < repeats; r++) {
            SourcePicker<CSRUWGraph> sp(&g);
            for (int i = 0; i < (r < 0 ? 1 : nsrc); i++) {
                nid_t s = sp.next_vertex();
                nid_t *parents = nullptr;
                const double t = bfs_do_cpu(g, s, &parents);
                if (r >= 0) ms.push_back(t);
                if (r == 0) {
                    sources.push_back(s);
                    write_out(out, parents, sizeof(nid_t) * (size_t)g.num_nodes);
                }
                delete[] parents;
            }
        }
    } else if (algo == "sssp" || algo == "sssp_dijkstra") {
        CSRWGraph g = load_graph_from_file<CSRWGraph>(path);
        n = g.num_nodes;
        m = g.num_edges;
        std::vector<weight_t> init(g.num_nodes, INF_WEIGHT);
        for (int r = -warmup; r < repeats; r++) {
            SourcePicker<CSRWGraph> sp(&g);
            for (int i = 0; i < (r < 0 ? 1 : nsrc); i++) {
                nid_t s = sp.next_vertex();
                weight_t *dist = nullptr;
                double t_ms = 0;
                if (algo == "sssp") {
                    init[s] = 0.0f;
                    t_ms = sssp_pull_cpu(g, epoch_sssp_pull_cpu_one_to_one, init.data(), &dist);
                    init[s] = INF_WEIGHT;
                } else {
                    Timer t;
                    t.Start();
                    sssp_dijkstras_cpu_serial(g, s, &dist);
                    t.Stop();
                    t_ms = t.Millisecs();
                }
                if (r >= 0) ms.push_back(t_ms);
                if (r == 0) {
                    sources.push_back(s);
                    write_out(out, dist, sizeof(weight_t) * (size_t)g.num_nodes);
                }
                delete[] dist;
            }
        }
    } else if (algo == "pr") {
        CSRWGraph g = load_graph_from_file<CSRWGraph>(path);
        n = g.num_nodes;
        m = g.num_edges;
        std::vector<weight_t> init(g.num_nodes, 1.0f / g.num_nodes);
        for (int r = -warmup; r < repeats; r++) {
            weight_t *score = nullptr;
            const double t = pr_pull_cpu(g, epoch_pr_pull_cpu_one_to_one, init.data(), &score);
            if (r >= 0) ms.push_back(t);
            if (r == 0) write_out(out, score, sizeof(weight_t) * (size_t)g.num_nodes);
            delete[] score;
        }
        iters = 0;
    } else {
        std::fprintf(stderr, "unknown algorithm %s\n", algo.c_str());
        return 1;
    }
    if (out) std::fclose(out);
    std::printf("{\"algo\": \"%s\", \"num_nodes\": %lld, \"num_edges\": %lld, \"threads\": %d, \"sources\": [",
                algo.c_str(), n, m, omp_get_max_threads());
    for (size_t i = 0; i < sources.size(); i++) std::printf("%s%d", i ? ", " : "", sources[i]);
    std::printf("], \"ms\": [");
    for (size_t i = 0; i < ms.size(); i++) std::printf("%s%.6f", i ? ", " : "", ms[i]);
    std::printf("], \"iters\": %d}\n", iters);
    return 0;
}
