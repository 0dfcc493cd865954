// Host side of the C ABI: error plumbing, synthetic graph construction,
// .sg/.wsg I/O and source picking.  No CUDA in this file.
//
// Graph construction restates the semantics of the reference's gapbs adapters
// (src/gapbs/generator.h:53-165, src/gapbs/builder.h:141-186 and :366-406):
// R-MAT quadrant recursion with A=.57 B=.19 C=.19, a random vertex-id
// permutation, symmetrisation, removal of self-loops and duplicate edges,
// relabelling by descending degree and sorted neighbour rows.  The random
// streams are this project's own (counter-based, thread-count independent);
// gapbs is not vendored in the reference, so its exact edge list is not
// reproduced -- the reference and this engine run on the same generated file.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <random>
#include <vector>

#include "hc_common.h"
#include "hc_gen.h"

namespace hc {

static thread_local std::string g_last_error;
static std::atomic<int64_t> g_launches{0};

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

hc_status fail(hc_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

void clear_error() { g_last_error.clear(); }

namespace {

hc_status alloc_csr(hc_csr *out, int32_t n, int64_t m, hc_wtype wt) {
    std::memset(out, 0, sizeof(*out));
    out->num_nodes = n;
    out->num_edges = m;
    out->wtype = wt;
    out->index = (int64_t *)std::malloc(sizeof(int64_t) * ((size_t)n + 1));
    out->neighbors = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
    if (wt != HC_W_NONE) out->weights = std::malloc(4 * (size_t)std::max<int64_t>(m, 1));
    if (!out->index || !out->neighbors || (wt != HC_W_NONE && !out->weights)) {
        hc_csr_free(out);
        return fail(HC_ERR_OOM, "host allocation of a %lld-edge CSR failed", (long long)m);
    }
    return HC_OK;
}

void exclusive_scan(const uint32_t *deg, int64_t *off, int64_t n) {
    // Two-level parallel scan.
    int nt = omp_get_max_threads();
    std::vector<int64_t> part(nt + 1, 0);
#pragma omp parallel num_threads(nt)
    {
        int t = omp_get_thread_num();
        int64_t lo = n * t / nt, hi = n * (t + 1) / nt, s = 0;
        for (int64_t i = lo; i < hi; i++) s += deg[i];
        part[t + 1] = s;
#pragma omp barrier
#pragma omp single
        for (int i = 0; i < nt; i++) part[i + 1] += part[i];
        s = part[t];
        for (int64_t i = lo; i < hi; i++) {
            off[i] = s;
            s += deg[i];
        }
    }
    off[n] = part[nt];
}

// Symmetrise, dedup, relabel by degree and emit the CSR.
template <class Pairs>
hc_status build_csr(const Pairs &pairs, int scale, int64_t num_pairs, hc_wtype wt,
                    uint64_t seed, hc_csr *out) {
    const int64_t n = 1ll << scale;
    if (n > 0x7fffffffll) return fail(HC_ERR_INVALID_ARG, "scale %d too large for int32 ids", scale);

    std::unique_ptr<std::atomic<uint32_t>[]> cnt(new std::atomic<uint32_t>[n]);
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; v++) cnt[v].store(0, std::memory_order_relaxed);

    // Pass 1: directed degree counts of the symmetrised list (no self-loops).
#pragma omp parallel for schedule(static, 1 << 16)
    for (int64_t e = 0; e < num_pairs; e++) {
        uint32_t s, d;
        pairs(e, s, d);
        if (s == d) continue;
        cnt[s].fetch_add(1, std::memory_order_relaxed);
        cnt[d].fetch_add(1, std::memory_order_relaxed);
    }
    std::vector<uint32_t> deg(n);
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; v++) {
        deg[v] = cnt[v].load(std::memory_order_relaxed);
        cnt[v].store(0, std::memory_order_relaxed);
    }
    std::vector<int64_t> off(n + 1);
    exclusive_scan(deg.data(), off.data(), n);
    const int64_t m_raw = off[n];

    // Pass 2: scatter packed (neighbour << 32 | weight bits) entries.
    uint64_t *packed = (uint64_t *)std::malloc(sizeof(uint64_t) * (size_t)std::max<int64_t>(m_raw, 1));
    if (!packed) return fail(HC_ERR_OOM, "host allocation of %lld edges failed", (long long)m_raw);
#pragma omp parallel for schedule(static, 1 << 16)
    for (int64_t e = 0; e < num_pairs; e++) {
        uint32_t s, d;
        pairs(e, s, d);
        if (s == d) continue;
        uint64_t w = weight_bits(wt, seed, e);
        int64_t ps = off[s] + cnt[s].fetch_add(1, std::memory_order_relaxed);
        int64_t pd = off[d] + cnt[d].fetch_add(1, std::memory_order_relaxed);
        packed[ps] = ((uint64_t)d << 32) | w;
        packed[pd] = ((uint64_t)s << 32) | w;
    }
    cnt.reset();

    // Pass 3: sort each row, keep the first (lightest) of each neighbour run.
    std::vector<uint32_t> ndeg(n);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; v++) {
        uint64_t *b = packed + off[v], *e = packed + off[v + 1];
        std::sort(b, e);
        uint64_t *o = b;
        for (uint64_t *p = b; p < e; p++)
            if (o == b || (o[-1] >> 32) != (*p >> 32)) *o++ = *p;
        ndeg[v] = (uint32_t)(o - b);
    }

    // Pass 4: new id = rank by (degree desc, old id desc), as the
    // std::greater sort of (degree, id) pairs in src/gapbs/builder.h:375-388.
    uint32_t maxdeg = 0;
    for (int64_t v = 0; v < n; v++) maxdeg = std::max(maxdeg, ndeg[v]);
    std::vector<int64_t> start((size_t)maxdeg + 2, 0);
    for (int64_t v = 0; v < n; v++) start[ndeg[v]]++;
    int64_t acc = 0;
    for (int64_t d = maxdeg; d >= 0; d--) {
        int64_t c = start[d];
        start[d] = acc;
        acc += c;
    }
    std::vector<int32_t> rank(n);
    for (int64_t v = n - 1; v >= 0; v--) rank[v] = (int32_t)(start[ndeg[v]]++);

    std::vector<uint32_t> deg_new(n);
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; v++) deg_new[rank[v]] = ndeg[v];
    std::vector<int64_t> noff(n + 1);
    exclusive_scan(deg_new.data(), noff.data(), n);
    const int64_t m = noff[n];

    // Pass 5: rows in the new order, neighbours renamed and re-sorted.
    uint64_t *tmp = (uint64_t *)std::malloc(sizeof(uint64_t) * (size_t)std::max<int64_t>(m, 1));
    if (!tmp) {
        std::free(packed);
        return fail(HC_ERR_OOM, "host allocation of %lld edges failed", (long long)m);
    }
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; v++) {
        const uint64_t *src = packed + off[v];
        uint64_t *dst = tmp + noff[rank[v]];
        for (uint32_t j = 0; j < ndeg[v]; j++) {
            uint64_t x = src[j];
            dst[j] = ((uint64_t)(uint32_t)rank[x >> 32] << 32) | (x & 0xffffffffull);
        }
    }
    std::free(packed);

    hc_status st = alloc_csr(out, (int32_t)n, m, wt);
    if (st != HC_OK) {
        std::free(tmp);
        return st;
    }
    std::memcpy(out->index, noff.data(), sizeof(int64_t) * (n + 1));
    uint32_t *wout = (uint32_t *)out->weights;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; v++) {
        uint64_t *b = tmp + noff[v], *e = tmp + noff[v + 1];
        std::sort(b, e);
        for (int64_t i = noff[v]; i < noff[v + 1]; i++) {
            out->neighbors[i] = (int32_t)(tmp[i] >> 32);
            if (wout) wout[i] = (uint32_t)tmp[i];
        }
    }
    std::free(tmp);
    return HC_OK;
}

bool read_exact(std::ifstream &is, void *p, size_t bytes) {
    is.read(reinterpret_cast<char *>(p), (std::streamsize)bytes);
    return (size_t)is.gcount() == bytes;
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" {

const char *hc_last_error(void) { return g_last_error.c_str(); }

const char *hc_status_string(hc_status s) {
    switch (s) {
        case HC_OK: return "ok";
        case HC_ERR_INVALID_ARG: return "invalid argument";
        case HC_ERR_OOM: return "out of memory";
        case HC_ERR_CUDA: return "CUDA error";
        case HC_ERR_NOT_CONVERGED: return "not converged";
        case HC_ERR_TIMEOUT: return "device wait timed out";
        case HC_ERR_NO_DEVICE: return "no CUDA device";
        case HC_ERR_UNSUPPORTED: return "unsupported";
        case HC_ERR_IO: return "I/O error";
    }
    return "unknown status";
}

int32_t hc_abi_version(void) { return 1; }

int64_t hc_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

void hc_csr_free(hc_csr *g) {
    if (!g) return;
    std::free(g->index);
    std::free(g->neighbors);
    std::free(g->weights);
    g->index = nullptr;
    g->neighbors = nullptr;
    g->weights = nullptr;
}

hc_status hc_gen_kronecker(int32_t scale, int32_t edge_factor, uint64_t seed,
                           hc_wtype wtype, hc_csr *out) {
    clear_error();
    if (!out || scale < 1 || scale > 30 || edge_factor < 1)
        return fail(HC_ERR_INVALID_ARG, "hc_gen_kronecker: bad scale %d / edge factor %d", scale, edge_factor);
    RmatPairs pairs(scale, seed);
    return build_csr(pairs, scale, (int64_t)edge_factor << scale, wtype, seed, out);
}

hc_status hc_gen_uniform(int32_t scale, int32_t degree, uint64_t seed, hc_wtype wtype,
                         hc_csr *out) {
    clear_error();
    if (!out || scale < 1 || scale > 30 || degree < 1)
        return fail(HC_ERR_INVALID_ARG, "hc_gen_uniform: bad scale %d / degree %d", scale, degree);
    UniformPairs pairs{scale, seed};
    return build_csr(pairs, scale, (int64_t)degree << scale, wtype, seed, out);
}

hc_status hc_gen_grid(int32_t rows, int32_t cols, uint64_t seed, hc_wtype wtype, hc_csr *out) {
    clear_error();
    if (!out || rows < 1 || cols < 1 || (int64_t)rows * cols > 0x7fffffffll)
        return fail(HC_ERR_INVALID_ARG, "hc_gen_grid: bad shape %d x %d", rows, cols);
    const int64_t n = (int64_t)rows * cols;
    const int64_t m = 2 * ((int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols);
    hc_status st = alloc_csr(out, (int32_t)n, m, wtype);
    if (st != HC_OK) return st;
    std::vector<uint32_t> deg(n);
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; v++) {
        int64_t r = v / cols, c = v % cols;
        deg[v] = (r > 0) + (c > 0) + (c + 1 < cols) + (r + 1 < rows);
    }
    exclusive_scan(deg.data(), out->index, n);
    uint32_t *w = (uint32_t *)out->weights;
    // Undirected edge ids: 2*v for (v, v+1), 2*v+1 for (v, v+cols); both
    // directions carry that edge's weight.  Neighbours come out sorted.
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; v++) {
        int64_t r = v / cols, c = v % cols, p = out->index[v];
        auto put = [&](int64_t u, int64_t eid) {
            out->neighbors[p] = (int32_t)u;
            if (w) w[p] = weight_bits(wtype, seed, eid);
            p++;
        };
        if (r > 0) put(v - cols, 2 * (v - cols) + 1);
        if (c > 0) put(v - 1, 2 * (v - 1));
        if (c + 1 < cols) put(v + 1, 2 * v);
        if (r + 1 < rows) put(v + cols, 2 * v + 1);
    }
    return HC_OK;
}

hc_status hc_csr_read(const char *path, int32_t weighted, hc_csr *out) {
    clear_error();
    if (!path || !out) return fail(HC_ERR_INVALID_ARG, "hc_csr_read: null argument");
    std::ifstream is(path, std::ios::binary);
    if (!is) return fail(HC_ERR_IO, "cannot open %s", path);
    int32_t n = 0;
    int64_t m = 0;
    if (!read_exact(is, &n, 4) || !read_exact(is, &m, 8) || n < 0 || m < 0)
        return fail(HC_ERR_IO, "%s: truncated or corrupt header", path);
    hc_wtype wt = weighted == 0 ? HC_W_NONE : (weighted == 2 ? HC_W_I32 : HC_W_F32);
    hc_status st = alloc_csr(out, n, m, wt);
    if (st != HC_OK) return st;
    if (!read_exact(is, out->index, sizeof(int64_t) * ((size_t)n + 1))) {
        hc_csr_free(out);
        return fail(HC_ERR_IO, "%s: truncated index", path);
    }
    if (out->index[0] != 0 || out->index[n] != m) {
        hc_csr_free(out);
        return fail(HC_ERR_IO, "%s: index does not span [0, %lld]", path, (long long)m);
    }
    for (int32_t v = 0; v < n; v++)
        if (out->index[v + 1] < out->index[v]) {
            hc_csr_free(out);
            return fail(HC_ERR_IO, "%s: index decreases at vertex %d", path, v);
        }
    if (wt == HC_W_NONE) {
        if (!read_exact(is, out->neighbors, sizeof(int32_t) * (size_t)m)) {
            hc_csr_free(out);
            return fail(HC_ERR_IO, "%s: truncated neighbour list", path);
        }
    } else {
        const size_t chunk = 1 << 20;
        std::vector<uint32_t> buf(2 * chunk);
        for (int64_t done = 0; done < m;) {
            size_t k = (size_t)std::min<int64_t>(chunk, m - done);
            if (!read_exact(is, buf.data(), 8 * k)) {
                hc_csr_free(out);
                return fail(HC_ERR_IO, "%s: truncated weighted neighbour list", path);
            }
            for (size_t i = 0; i < k; i++) {
                out->neighbors[done + i] = (int32_t)buf[2 * i];
                float f;
                std::memcpy(&f, &buf[2 * i + 1], 4);
                if (wt == HC_W_F32) {
                    ((float *)out->weights)[done + i] = f;
                } else {
                    if (!(f >= 0.f && f <= 2147483520.f) || std::floor(f) != f) {
                        hc_csr_free(out);
                        return fail(HC_ERR_IO, "%s: weight %g is not a non-negative integer", path, f);
                    }
                    ((int32_t *)out->weights)[done + i] = (int32_t)f;
                }
            }
            done += (int64_t)k;
        }
    }
    for (int64_t i = 0; i < m; i++)
        if (out->neighbors[i] < 0 || out->neighbors[i] >= n) {
            const int32_t bad = out->neighbors[i];
            hc_csr_free(out);
            return fail(HC_ERR_IO, "%s: neighbour %d out of range at edge %lld", path, bad, (long long)i);
        }
    return HC_OK;
}

hc_status hc_csr_write(const char *path, const hc_csr *g) {
    clear_error();
    if (!path || !g || !g->index || (!g->neighbors && g->num_edges))
        return fail(HC_ERR_INVALID_ARG, "hc_csr_write: null argument");
    std::ofstream os(path, std::ios::binary);
    if (!os) return fail(HC_ERR_IO, "cannot create %s", path);
    os.write(reinterpret_cast<const char *>(&g->num_nodes), 4);
    os.write(reinterpret_cast<const char *>(&g->num_edges), 8);
    os.write(reinterpret_cast<const char *>(g->index), 8 * ((size_t)g->num_nodes + 1));
    if (g->wtype == HC_W_NONE || !g->weights) {
        // 4 bytes per edge; the reference's gapbs writer wrote 8 (the over-read
        // at src/gapbs/gapbs.cuh:79-80), which its loader then ignored.
        os.write(reinterpret_cast<const char *>(g->neighbors), 4 * (size_t)g->num_edges);
    } else {
        const size_t chunk = 1 << 20;
        std::vector<uint32_t> buf(2 * chunk);
        for (int64_t done = 0; done < g->num_edges;) {
            size_t k = (size_t)std::min<int64_t>(chunk, g->num_edges - done);
            for (size_t i = 0; i < k; i++) {
                buf[2 * i] = (uint32_t)g->neighbors[done + i];
                float f = g->wtype == HC_W_F32 ? ((const float *)g->weights)[done + i]
                                               : (float)((const int32_t *)g->weights)[done + i];
                std::memcpy(&buf[2 * i + 1], &f, 4);
            }
            os.write(reinterpret_cast<const char *>(buf.data()), 8 * k);
            done += (int64_t)k;
        }
    }
    if (!os) return fail(HC_ERR_IO, "write to %s failed", path);
    return HC_OK;
}

hc_status hc_equal_edge_ranges(const int64_t *index, int32_t num_nodes, int32_t num_segments, int32_t chunk_size,
                               int32_t *ranges_out) {
    clear_error();
    if (!index || !ranges_out || num_nodes < 1 || num_segments < 1 || chunk_size < 1)
        return fail(HC_ERR_INVALID_ARG, "hc_equal_edge_ranges: bad arguments");
    const int64_t m = index[num_nodes] - index[0];
    const int64_t avg = m / num_segments;
    ranges_out[0] = 0;
    int32_t seg = 0;
    int64_t acc = 0;
    int32_t v = 0;
    for (; v < num_nodes; v++) {
        acc += index[v + 1] - index[v];
        if (acc >= avg && seg + 1 < num_segments) {  // the reference has no bound on seg here
            ranges_out[seg + 1] = v;
            acc = 0;
            seg++;
        }
    }
    for (int32_t s = seg + 1; s <= num_segments; s++) ranges_out[s] = num_nodes;
    for (int32_t s = 1; s < num_segments; s++) {
        const int32_t r = ranges_out[s] % chunk_size;
        if (r != 0) ranges_out[s] = r < chunk_size / 2 ? ranges_out[s] - r : std::min(ranges_out[s] - r + chunk_size, num_nodes);
    }
    return HC_OK;
}

hc_status hc_pick_sources(const int64_t *index, const int32_t *neighbors, int32_t num_nodes,
                          int32_t count, int32_t const_source, int32_t *out) {
    clear_error();
    if (!index || !out || num_nodes < 1 || count < 0)
        return fail(HC_ERR_INVALID_ARG, "hc_pick_sources: bad arguments");
    // A degree-1 vertex whose only edge is a self-loop is no source.
    auto self_only = [&](int32_t v) { return neighbors && neighbors[index[v]] == v; };
    return pick_sources_impl(index, num_nodes, count, const_source, out, self_only);
}

}  // extern "C"
