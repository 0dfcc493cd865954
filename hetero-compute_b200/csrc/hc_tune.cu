// Autotuner: times candidate launch parameters on the caller's sample sources
// and keeps the fastest on the graph handle (hc_graph::tune).  Every trial is
// a normal call through the C ABI with its outputs discarded, timed by the
// call's own CUDA events (stats.ms), so a trial runs exactly the code a later
// call will.  The search is coordinate descent: one parameter at a time, all
// of its candidates with the others held at their current values, keeping a
// candidate only when it beats the current value by more than kKeepMargin.
//
// The reference has no counterpart: its variant and launch shape are picked
// by hand per call (src/kernels/gpu/bfs.cuh:352-360, sssp.cuh:343-351).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr double kKeepMargin = 0.02;
constexpr double kFailed = std::numeric_limits<double>::infinity();

struct Tuner {
    hc_graph *g;
    std::vector<int32_t> src;
    int trials = 0;
    double ms = 0;

    // Device milliseconds per source of one call, or kFailed when the
    // candidate cannot run (e.g. a group too wide for free memory).
    double bfs(const hc_bfs_opts &o, int k) {
        hc_bfs_stats st{};
        if (hc_bfs(g, src.data(), k, nullptr, nullptr, &o, &st) != HC_OK) return kFailed;
        return note(st.ms, k);
    }
    double sssp(const hc_sssp_opts &o, int k) {
        hc_sssp_stats st{};
        if (hc_sssp(g, src.data(), k, nullptr, nullptr, &o, &st) != HC_OK) return kFailed;
        return note(st.ms, k);
    }
    double bfs_batched(const hc_batch_opts &o, int k) {
        hc_batch_stats st{};
        if (hc_bfs_batched(g, src.data(), k, nullptr, &o, &st) != HC_OK) return kFailed;
        return note(st.ms, k);
    }
    double sssp_batched(const hc_batch_opts &o, int k) {
        hc_batch_stats st{};
        if (hc_sssp_batched(g, src.data(), k, nullptr, &o, &st) != HC_OK) return kFailed;
        return note(st.ms, k);
    }
    double note(double t, int k) {
        trials++;
        ms += t;
        return t / k;
    }
};

// Tries every value of `cands` for the field `*field` of `opts`, starting
// from `*field` (whose time is `best`), and leaves the winner in `*field`.
template <class Opts, class Run>
void descend(Opts &opts, int32_t *field, const std::vector<int32_t> &cands, double &best, Run &&run) {
    const int32_t start = *field;
    int32_t keep = start;
    for (int32_t c : cands) {
        if (c == start) continue;
        *field = c;
        const double t = run(opts);
        if (t < best * (1.0 - kKeepMargin)) {
            best = t;
            keep = c;
        }
    }
    *field = keep;
}

hc_status tune_bfs(Tuner &tu, hc_tuning &out) {
    const int k = (int)std::min<size_t>(tu.src.size(), 32);
    hc_bfs_opts o{};
    o.alpha = out.bfs_alpha > 0 ? out.bfs_alpha : 15;
    o.beta = out.bfs_beta > 0 ? out.bfs_beta : 18;
    o.bu_variant = out.bfs_bu_variant > 0 ? (hc_variant)out.bfs_bu_variant : HC_VARIANT_THREAD;
    auto run = [&](const hc_bfs_opts &x) { return tu.bfs(x, k); };
    tu.bfs(o, 1);  // warm-up: workspaces and plans
    double best = run(o);
    if (best == kFailed) return fail(HC_ERR_CUDA, "hc_autotune: BFS trial failed");
    int32_t var = (int32_t)o.bu_variant;
    {
        const int32_t start = var;
        for (int32_t c : {1, 2, 3}) {
            if (c == start) continue;
            o.bu_variant = (hc_variant)c;
            const double t = run(o);
            if (t < best * (1.0 - kKeepMargin)) {
                best = t;
                var = c;
            }
        }
        o.bu_variant = (hc_variant)var;
    }
    // Cheap sparse bottom-up levels (frontier summaries) make an early switch
    // pay on large graphs: the range reaches well above the reference's 15.
    descend(o, &o.alpha, {4, 8, 15, 30, 45, 60, 90, 120, 240}, best, run);
    {
        std::vector<int32_t> fine;
        for (double f : {0.7, 1.4}) fine.push_back((int32_t)std::max(1.0, std::floor(o.alpha * f)));
        descend(o, &o.alpha, fine, best, run);
    }
    descend(o, &o.beta, {6, 12, 18, 36, 72}, best, run);
    out.bfs_alpha = o.alpha;
    out.bfs_beta = o.beta;
    out.bfs_bu_variant = (int32_t)o.bu_variant;
    return HC_OK;
}

// The per-epoch granularity selector of bottom-up BFS: for each bottom-up
// level in turn (up to HC_BFS_SPLIT_LEVELS, as many as the sample runs have),
// the warp/thread split point is searched among the 32-aligned bounds of
// equal-edge vertex segments (hc_equal_edge_ranges, the reference's
// compute_equal_edge_ranges segmentation), the other levels held at their
// current split, whole BFS calls timed.  The table is kept only if some level
// moved off the tuned variant's fixed split.
hc_status tune_bfs_levels(Tuner &tu, hc_tuning &out) {
    hc_graph *g = tu.g;
    const int k = (int)std::min<size_t>(tu.src.size(), 16);
    hc_bfs_opts o{};
    o.alpha = out.bfs_alpha > 0 ? out.bfs_alpha : 15;
    o.beta = out.bfs_beta > 0 ? out.bfs_beta : 18;
    const int var = out.bfs_bu_variant > 0 ? out.bfs_bu_variant : HC_VARIANT_THREAD;
    const int32_t base = var == HC_VARIANT_WARP ? g->n_active : (var == HC_VARIANT_BLOCK ? g->n_warp_rows : 0);
    // Bottom-up levels per run on the samples.
    o.bu_variant = (hc_variant)var;
    hc_bfs_stats st{};
    HC_TRY(hc_bfs(g, tu.src.data(), k, nullptr, nullptr, &o, &st));
    const int levels = std::min(HC_BFS_SPLIT_LEVELS, (st.bu_levels + k - 1) / std::max(k, 1));
    if (levels < 1) return HC_OK;
    // Candidates: 32-aligned bounds of 16 equal-edge segments of the active rows.
    std::vector<int64_t> index((size_t)g->N + 1);
    HC_CUDA_TRY(cudaMemcpyAsync(index.data(), g->index.ptr, sizeof(int64_t) * index.size(), cudaMemcpyDeviceToHost,
                                g->stream));
    HC_CUDA_TRY(cudaStreamSynchronize(g->stream));
    std::vector<int32_t> bounds(17);
    HC_TRY(hc_equal_edge_ranges(index.data(), std::max(g->n_active, 1), 16, 32, bounds.data()));
    std::vector<int32_t> cands(bounds.begin(), bounds.end());
    cands.push_back(g->n_warp_rows);
    std::sort(cands.begin(), cands.end());
    cands.erase(std::unique(cands.begin(), cands.end()), cands.end());

    hc_tuning &live = g->tune;  // trials read the table from the handle (bu_variant AUTO)
    live.bfs_bu_variant = var;
    live.bfs_bu_split_levels = levels;
    for (int l = 0; l < levels; l++) live.bfs_bu_split[l] = base;
    o.bu_variant = HC_VARIANT_AUTO;
    auto run = [&](const hc_bfs_opts &x) { return tu.bfs(x, k); };
    double best = run(o);
    if (best == kFailed) return fail(HC_ERR_CUDA, "hc_autotune: BFS level trial failed");
    bool moved = false;
    for (int l = 0; l < levels; l++) {
        descend(o, &live.bfs_bu_split[l], cands, best, run);
        moved |= live.bfs_bu_split[l] != base;
    }
    if (moved) {
        out.bfs_bu_split_levels = levels;
        for (int l = 0; l < HC_BFS_SPLIT_LEVELS; l++) out.bfs_bu_split[l] = l < levels ? live.bfs_bu_split[l] : 0;
    } else {
        out.bfs_bu_split_levels = 0;
    }
    live.bfs_bu_split_levels = 0;
    live.bfs_bu_variant = 0;
    return HC_OK;
}

hc_status tune_sssp(Tuner &tu, hc_tuning &out) {
    hc_graph *g = tu.g;
    if (g->wtype != HC_W_I32) return HC_OK;  // no SSSP on this graph
    HC_TRY(ensure_weight_stats(g));
    if (g->w_negative) return HC_OK;
    // 16 sample sources: the push/pull and delta choices move the time by a
    // few percent, about what the spread between 8 sources is.
    const int k = (int)std::min<size_t>(tu.src.size(), 16);
    // The built-in delta (hc_sssp): mean weight x 32 / mean degree.
    const double davg = g->n_active ? (double)g->M / (double)g->n_active : 1.0;
    const int32_t base = (int32_t)std::max(1.0, std::min(1e9, g->w_mean * 32.0 / std::max(davg, 1.0)));
    hc_sssp_opts o{};
    o.delta = out.sssp_delta > 0 ? out.sssp_delta : base;
    o.pull_alpha = out.sssp_pull_alpha != 0 ? out.sssp_pull_alpha : 10;
    auto run = [&](const hc_sssp_opts &x) { return tu.sssp(x, k); };
    tu.sssp(o, 1);
    double best = run(o);
    if (best == kFailed) return fail(HC_ERR_CUDA, "hc_autotune: SSSP trial failed");
    std::vector<int32_t> deltas;
    for (double f : {0.25, 0.5, 1.0, 2.0, 4.0}) deltas.push_back((int32_t)std::max(1.0, std::floor(base * f)));
    descend(o, &o.delta, deltas, best, run);
    if (g->w_symmetric) descend(o, &o.pull_alpha, {2, 4, 6, 8, 10, 12, 16, -1}, best, run);
    // Second, finer pass around the winners.
    std::vector<int32_t> fine;
    for (double f : {0.7, 0.85, 1.2, 1.4}) fine.push_back((int32_t)std::max(1.0, std::floor(o.delta * f)));
    descend(o, &o.delta, fine, best, run);
    if (g->w_symmetric && o.pull_alpha > 0) {
        std::vector<int32_t> near;
        for (int32_t x : {o.pull_alpha - 1, o.pull_alpha + 1, o.pull_alpha * 3 / 2})
            if (x >= 1) near.push_back(x);
        descend(o, &o.pull_alpha, near, best, run);
    }
    out.sssp_delta = o.delta;
    out.sssp_pull_alpha = o.pull_alpha;
    // Blocks per SM of the persistent kernel (read from the handle by the
    // launch; the trials set it there).
    g->tune.sssp_blocks_per_sm = 0;
    int32_t bps = 0;
    descend(o, &g->tune.sssp_blocks_per_sm, {1}, best, run);
    bps = g->tune.sssp_blocks_per_sm;
    g->tune.sssp_blocks_per_sm = 0;
    out.sssp_blocks_per_sm = bps;
    return HC_OK;
}

hc_status tune_bfs_batched(Tuner &tu, hc_tuning &out) {
    const int k = (int)std::min<size_t>(tu.src.size(), 512);
    hc_batch_opts o{};
    o.group = out.mbfs_group > 0 ? out.mbfs_group : 512;
    o.switch_alpha = out.mbfs_switch_alpha != 0 ? out.mbfs_switch_alpha : 10;
    auto run = [&](const hc_batch_opts &x) { return tu.bfs_batched(x, k); };
    tu.bfs_batched(o, std::min(k, 64));
    double best = run(o);
    if (best == kFailed) return fail(HC_ERR_CUDA, "hc_autotune: batched BFS trial failed");
    descend(o, &o.group, {64, 128, 256, 512}, best, run);
    descend(o, &o.switch_alpha, {5, 10, 20, 40, -1}, best, run);
    out.mbfs_group = o.group;
    out.mbfs_switch_alpha = o.switch_alpha;
    return HC_OK;
}

hc_status tune_sssp_batched(Tuner &tu, hc_tuning &out) {
    hc_graph *g = tu.g;
    if (g->wtype != HC_W_I32) return HC_OK;
    HC_TRY(ensure_weight_stats(g));
    if (g->w_negative) return HC_OK;
    const int k = (int)std::min<size_t>(tu.src.size(), 512);
    // Widest group that fits, as hc_sssp_batched picks it untuned.
    size_t free_b = 0, total_b = 0;
    HC_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    free_b += g->ws_batch.bytes + g->ws_out0.bytes;
    std::vector<int32_t> groups;
    const double bytes = g->w_max <= kMsspNarrowMaxW ? 2.0 : 4.0;  // 16- or 32-bit distances
    for (int32_t w : {64, 128, 256, 512})
        if ((double)g->N * w * bytes <= 0.4 * (double)free_b) groups.push_back(w);
    if (groups.empty()) groups.push_back(32);
    hc_batch_opts o{};
    o.group = out.mssp_group > 0 ? out.mssp_group : groups.back();
    o.switch_alpha = out.mssp_switch_alpha != 0 ? out.mssp_switch_alpha : 2;
    auto run = [&](const hc_batch_opts &x) { return tu.sssp_batched(x, k); };
    tu.sssp_batched(o, std::min(k, 32));
    double best = run(o);
    if (best == kFailed) return fail(HC_ERR_CUDA, "hc_autotune: batched SSSP trial failed");
    descend(o, &o.group, groups, best, run);
    if (g->w_symmetric) descend(o, &o.switch_alpha, {1, 2, 4, -1}, best, run);
    out.mssp_group = o.group;
    out.mssp_switch_alpha = o.switch_alpha;
    return HC_OK;
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_autotune(hc_graph *g, const int32_t *sample_sources, int32_t num_samples, uint32_t what,
                                 hc_tuning *out) {
    clear_error();
    HC_TRY(activate(g));
    if (!sample_sources || num_samples < 1) return fail(HC_ERR_INVALID_ARG, "hc_autotune: no sample sources");
    if (what & ~HC_TUNE_ALL) return fail(HC_ERR_INVALID_ARG, "hc_autotune: unknown target bits 0x%x", what);
    Tuner tu{g};
    tu.src.resize(num_samples);
    HC_CUDA_TRY(cudaMemcpy(tu.src.data(), sample_sources, sizeof(int32_t) * num_samples, cudaMemcpyDefault));
    for (int32_t s : tu.src)
        if (s < 0 || s >= g->N) return fail(HC_ERR_INVALID_ARG, "hc_autotune: source %d out of range", s);
    // Trials run with the handle's tuning cleared for the fields being
    // searched, so that the explicit candidate values are what run.
    hc_tuning t = g->tune;
    const hc_tuning saved = g->tune;
    std::memset(&g->tune, 0, sizeof(g->tune));
    hc_status st = HC_OK;
    if (st == HC_OK && (what & HC_TUNE_BFS)) st = tune_bfs(tu, t);
    if (st == HC_OK && (what & HC_TUNE_BFS_LEVELS)) st = tune_bfs_levels(tu, t);
    if (st == HC_OK && (what & HC_TUNE_SSSP)) st = tune_sssp(tu, t);
    if (st == HC_OK && (what & HC_TUNE_BFS_BATCHED)) st = tune_bfs_batched(tu, t);
    if (st == HC_OK && (what & HC_TUNE_SSSP_BATCHED)) st = tune_sssp_batched(tu, t);
    if (st != HC_OK) {
        g->tune = saved;
        return st;
    }
    t.trials = tu.trials;
    t.tune_ms = tu.ms;
    g->tune = t;
    if (out) *out = t;
    return HC_OK;
}

extern "C" hc_status hc_get_tuning(const hc_graph *g, hc_tuning *out) {
    clear_error();
    if (!g || !out) return fail(HC_ERR_INVALID_ARG, "hc_get_tuning: null argument");
    *out = g->tune;
    return HC_OK;
}

extern "C" hc_status hc_set_tuning(hc_graph *g, const hc_tuning *t) {
    clear_error();
    if (!g || !t) return fail(HC_ERR_INVALID_ARG, "hc_set_tuning: null argument");
    if (t->bfs_bu_variant < 0 || t->bfs_bu_variant > 3)
        return fail(HC_ERR_INVALID_ARG, "hc_set_tuning: bad BFS variant %d", t->bfs_bu_variant);
    if (t->bfs_alpha < 0 || t->bfs_beta < 0 || t->mbfs_group < 0 || t->mssp_group < 0)
        return fail(HC_ERR_INVALID_ARG, "hc_set_tuning: negative threshold or group");
    if (t->sssp_blocks_per_sm < 0) return fail(HC_ERR_INVALID_ARG, "hc_set_tuning: negative blocks per SM");
    if (t->bfs_bu_split_levels < 0 || t->bfs_bu_split_levels > HC_BFS_SPLIT_LEVELS)
        return fail(HC_ERR_INVALID_ARG, "hc_set_tuning: bad split level count %d", t->bfs_bu_split_levels);
    for (int l = 0; l < t->bfs_bu_split_levels; l++)
        if (t->bfs_bu_split[l] < 0 || t->bfs_bu_split[l] > g->N)
            return fail(HC_ERR_INVALID_ARG, "hc_set_tuning: split %d outside [0, N]", t->bfs_bu_split[l]);
    g->tune = *t;
    return HC_OK;
}
