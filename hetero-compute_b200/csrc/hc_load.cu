// .sg / .wsg files streamed straight into a device graph.
//
// The reference's loader (src/graph.cuh:207-239) reads the whole file into
// host arrays, and its drivers copy those to the GPU on every call
// (src/kernels/gpu/sssp.cuh:51-61).  hc_graph_load reads the file in chunks
// through two pinned staging buffers: while one chunk's copy runs on the
// handle's stream, the next chunk is read from the file into the other
// buffer, so disk reads overlap host-to-device copies and host memory stays
// at two chunks whatever the graph's size.  Offsets and (.sg) neighbour ids
// land in place; the interleaved {int32 v; float w} records of a .wsg file
// land in a device staging chunk and a kernel splits them into the separate
// neighbour and weight arrays (checking integer weights when asked to convert
// them).  The handle is then validated and analysed like one from
// hc_graph_create.
#include <cstdio>
#include <cstring>

#include "hc_graph.cuh"

namespace hc {
namespace {

constexpr size_t kLoadChunk = 32u << 20;  // bytes per staging buffer

// Splits n {v, w} records into neighbours and weights.  to_int: the weights
// must be non-negative integers below 2^31 and are stored as int32; bit 0 of
// *bad records one that is not.
__global__ void split_records(const uint32_t *rec, int64_t n, int32_t *nbr, uint32_t *w, int to_int, int *bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint2 r = reinterpret_cast<const uint2 *>(rec)[i];
        nbr[i] = (int32_t)r.x;
        if (to_int) {
            const float f = __uint_as_float(r.y);
            const bool ok = f >= 0.f && f <= 2147483520.f && truncf(f) == f;
            if (!ok) atomicOr(bad, 1);
            w[i] = ok ? (uint32_t)(int32_t)f : 0u;
        } else {
            w[i] = r.y;
        }
    }
}

struct Stager {
    hc_graph *g;
    FILE *f;
    PinnedBuf host[2];
    cudaEvent_t done[2] = {nullptr, nullptr};
    int next = 0;
    ~Stager() {
        for (int i = 0; i < 2; i++) {
            if (done[i]) cudaEventDestroy(done[i]);
            host[i].release();
        }
    }
    hc_status init() {
        for (int i = 0; i < 2; i++) {
            HC_TRY(host[i].ensure(kLoadChunk));
            HC_CUDA_TRY(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
        }
        return HC_OK;
    }
    // Reads `bytes` from the file into the next staging buffer (after its last
    // copy finished) and copies them to dst on the handle's stream.
    hc_status chunk(void *dst, size_t bytes, const char *path) {
        const int b = next;
        next ^= 1;
        HC_CUDA_TRY(cudaEventSynchronize(done[b]));
        if (std::fread(host[b].ptr, 1, bytes, f) != bytes) return fail(HC_ERR_IO, "%s: file is truncated", path);
        HC_CUDA_TRY(cudaMemcpyAsync(dst, host[b].ptr, bytes, cudaMemcpyHostToDevice, g->stream));
        HC_CUDA_TRY(cudaEventRecord(done[b], g->stream));
        return HC_OK;
    }
    // Streams `bytes` from the file to device memory at dst.
    hc_status stream(char *dst, size_t bytes, const char *path) {
        for (size_t off = 0; off < bytes; off += kLoadChunk) HC_TRY(chunk(dst + off, std::min(kLoadChunk, bytes - off), path));
        return HC_OK;
    }
};

hc_status load(const char *path, int32_t weighted, int32_t device, hc_graph **out) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(HC_ERR_IO, "cannot open %s", path);
    struct Closer {
        FILE *f;
        ~Closer() { std::fclose(f); }
    } closer{f};
    int32_t n = 0;
    int64_t m = 0;
    if (std::fread(&n, 4, 1, f) != 1 || std::fread(&m, 8, 1, f) != 1 || n < 1 || m < 0)
        return fail(HC_ERR_IO, "%s: truncated or corrupt header", path);
    // The file must hold the records the header announces (bytes after them
    // are ignored, as the reference's loader ignores them).
    const size_t rec = weighted ? 8 : 4;
    const long long want = 12 + 8ll * ((long long)n + 1) + (long long)rec * m;
    if (std::fseek(f, 0, SEEK_END) != 0) return fail(HC_ERR_IO, "%s: cannot seek", path);
    const long long size = std::ftell(f);
    if (size < want)
        return fail(HC_ERR_IO, "%s: %lld bytes, the header (N=%d, M=%lld) needs %lld", path, size, n, (long long)m,
                    want);
    if (std::fseek(f, 12, SEEK_SET) != 0) return fail(HC_ERR_IO, "%s: cannot seek", path);

    const hc_wtype wt = weighted == 0 ? HC_W_NONE : (weighted == 2 ? HC_W_I32 : HC_W_F32);
    hc_graph *g = nullptr;
    HC_TRY(graph_alloc(n, m, wt, device, &g));
    auto bail = [&](hc_status s) {
        cudaStreamSynchronize(g->stream);
        hc_graph_destroy(g);
        return s;
    };
    hc_status st;
    {
        Stager sg{g, f};
        if ((st = sg.init()) != HC_OK) return bail(st);
        if ((st = sg.stream(g->index.as<char>(), 8 * ((size_t)n + 1), path)) != HC_OK) return bail(st);
        if (!weighted) {
            if ((st = sg.stream(g->nbr.as<char>(), 4 * (size_t)m, path)) != HC_OK) return bail(st);
        } else {
            // Records go through two device chunks; the split of chunk i runs
            // on the stream after its copy, so a chunk is reused only once the
            // split that read it is done (stream order).
            DevBuf staging[2], bad;
            if ((st = staging[0].ensure(kLoadChunk)) != HC_OK || (st = staging[1].ensure(kLoadChunk)) != HC_OK ||
                (st = bad.ensure(sizeof(int))) != HC_OK)
                return bail(st);
            if (cudaMemsetAsync(bad.ptr, 0, sizeof(int), g->stream) != cudaSuccess)
                return bail(fail(HC_ERR_CUDA, "memset failed"));
            const int64_t per = (int64_t)(kLoadChunk / 8);
            int i = 0;
            for (int64_t e0 = 0; e0 < m; e0 += per, i ^= 1) {
                const int64_t k = std::min(per, m - e0);
                if ((st = sg.chunk(staging[i].ptr, 8 * (size_t)k, path)) != HC_OK) return bail(st);
                const int blocks = (int)std::min<int64_t>((int64_t)g->sm_count * 8, (k + 255) / 256);
                split_records<<<blocks, 256, 0, g->stream>>>(staging[i].as<uint32_t>(), k, g->nbr.as<int32_t>() + e0,
                                                             g->wgt.as<uint32_t>() + e0, wt == HC_W_I32, bad.as<int>());
                count_launch();
                if (cudaGetLastError() != cudaSuccess) return bail(fail(HC_ERR_CUDA, "split_records launch failed"));
            }
            int h = 0;
            if (cudaMemcpyAsync(&h, bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
                cudaStreamSynchronize(g->stream) != cudaSuccess)
                return bail(fail(HC_ERR_CUDA, "%s: load failed", path));
            if (h) return bail(fail(HC_ERR_IO, "%s: a weight is not a non-negative integer below 2^31", path));
        }
        if (cudaStreamSynchronize(g->stream) != cudaSuccess) return bail(fail(HC_ERR_CUDA, "%s: load failed", path));
    }
    if ((st = graph_finish(g, "hc_graph_load")) != HC_OK) {
        hc_graph_destroy(g);
        return st == HC_ERR_INVALID_ARG ? fail(HC_ERR_IO, "%s: %s", path, hc_last_error()) : st;
    }
    *out = g;
    return HC_OK;
}

}  // namespace
}  // namespace hc

extern "C" hc_status hc_graph_load(const char *path, int32_t weighted, int32_t device, hc_graph **out) {
    hc::clear_error();
    if (!path || !out || weighted < 0 || weighted > 2)
        return hc::fail(HC_ERR_INVALID_ARG, "hc_graph_load: bad arguments");
    *out = nullptr;
    return hc::load(path, weighted, device, out);
}
