// Device-side building blocks shared by the BFS / SSSP / PageRank kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "hc_common.h"

#define HC_CUDA_TRY(expr)                                                        \
    do {                                                                         \
        cudaError_t _e = (expr);                                                 \
        if (_e != cudaSuccess)                                                   \
            return ::hc::fail(_e == cudaErrorMemoryAllocation ? HC_ERR_OOM      \
                                                               : HC_ERR_CUDA,   \
                              "%s failed: %s (%s:%d)", #expr,                    \
                              cudaGetErrorString(_e), __FILE__, __LINE__);       \
    } while (0)

#define HC_TRY(expr)                        \
    do {                                    \
        hc_status _s = (expr);              \
        if (_s != HC_OK) return _s;         \
    } while (0)

namespace hc {

constexpr unsigned kFull = 0xffffffffu;
constexpr int32_t kInfDist = 0x7fffffff;

// Time limits of the device-side waits (defaults below; hc_set_time_limits
// shortens them so that tests can make each one run out):
//   wait  every device-side spin: a wait that lasts longer gives up, records
//         HC_ERR_TIMEOUT and lets the kernel return;
//   run   one persistent run (all its epochs): past it the run records
//         HC_ERR_TIMEOUT and every block leaves at the next barrier;
//   loop  one batched group's epoch loop (a CUDA-graph while loop), checked
//         by the kernel that ends each epoch.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;
constexpr unsigned long long kRunLimitNs = 20000000000ull;
constexpr unsigned long long kLoopLimitNs = 60000000000ull;
struct TimeLimits {
    unsigned long long wait_ns, run_ns, loop_ns;
};
// One copy per translation unit (no relocatable device code); every copy is
// registered with the setter behind hc_set_time_limits.
static __constant__ TimeLimits c_limits = {kWaitLimitNs, kRunLimitNs, kLoopLimitNs};
using LimitSetter = hc_status (*)(const TimeLimits &);
void register_limit_setter(LimitSetter f);
static hc_status set_unit_limits(const TimeLimits &t) {
    if (cudaMemcpyToSymbol(c_limits, &t, sizeof(t)) != cudaSuccess)
        return fail(HC_ERR_CUDA, "hc_set_time_limits: cudaMemcpyToSymbol failed");
    return HC_OK;
}
namespace {
struct LimitSetterReg {
    LimitSetterReg() { register_limit_setter(&set_unit_limits); }
};
static LimitSetterReg g_limit_setter_reg;
}  // namespace

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier for cooperative (co-resident) launches.  `count` only
// grows: every block adds one per barrier, so barrier k of a run is complete
// when count reaches (k + 1) * gridDim.x, and a block computes that target
// from the value its own arrival returned; no block resets anything, and the
// waiters see the last arrival itself.  The control block must be zeroed
// before a run, and every launch of a run must use the same grid size.
// Waiters poll `count` with an acquire load and give up after the wait
// limit, setting *err.  Once *err is set every later barrier returns at once,
// so a failed run drains in bounded time.  Returns false when the run must
// stop.
struct GridSync {
    unsigned long long count;
    int err;
    int pad;
};

__device__ __forceinline__ bool grid_barrier(GridSync *gs) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        if (*(volatile int *)&gs->err) {
            ok = 0;
        } else {
            __threadfence();
            const unsigned long long t = atomicAdd(&gs->count, 1ull);
            const unsigned long long target = (t / gridDim.x + 1) * gridDim.x;
            if (t + 1 != target) {
                unsigned long long t0 = globaltimer_ns();
                while (ld_acquire_u64(&gs->count) < target) {
                    if (*(volatile int *)&gs->err) { ok = 0; break; }
                    if (globaltimer_ns() - t0 > c_limits.wait_ns) {
                        atomicExch(&gs->err, (int)HC_ERR_TIMEOUT);
                        ok = 0;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            __threadfence();
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Warp-level helpers (full mask; the reference's ALLWARP mask at
// src/cuda.cuh:24 evaluates to 0x80000000, which is not a full warp).
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}
template <class T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
// Exclusive prefix sum across the warp; *total receives the warp total.
template <class T>
__device__ __forceinline__ T warp_exclusive_scan(T v, T *total) {
    const int lane = threadIdx.x & 31;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    *total = __shfl_sync(kFull, x, 31);
    return x - v;
}

// Block-wide sum of a per-thread value (blockDim.x a multiple of 32, <= 1024).
template <class T>
__device__ __forceinline__ T block_sum(T v, T *smem32) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) smem32[w] = v;
    __syncthreads();
    T r = 0;
    if (w == 0) {
        r = lane < (int)(blockDim.x >> 5) ? smem32[lane] : T(0);
        r = warp_sum(r);
    }
    return r;  // valid in thread 0
}

// L2-coherent loads for state that other blocks write during a launch.
__device__ __forceinline__ int32_t ld_cg(const int32_t *p) { return __ldcg(p); }
__device__ __forceinline__ uint32_t ld_cg(const uint32_t *p) { return __ldcg(p); }

// ------------------------------------------------------------- host helpers

// True when `p` is device (or managed) memory of the current context.
bool is_device_pointer(const void *p);

// Device buffer that grows on demand and is freed with its owner (or when it
// goes out of scope; not copyable).
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    hc_status ensure(size_t want);
    void release();
    template <class T>
    T *as() const { return reinterpret_cast<T *>(ptr); }
};

// Pinned host buffer that grows on demand.
struct PinnedBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    hc_status ensure(size_t want);
    void release();
    template <class T>
    T *as() const { return reinterpret_cast<T *>(ptr); }
};

// Copies between user memory (host or device) and HBM on `s`.
hc_status copy_in(void *dst_dev, const void *src_any, size_t bytes, cudaStream_t s);
hc_status copy_out(void *dst_any, const void *src_dev, size_t bytes, cudaStream_t s);

// An epoch loop as a CUDA graph: one conditional while node whose body is
// captured from `body(stream, handle)`.  The body's last kernel sets the
// condition with cudaGraphSetConditional; the handle starts at 1 on every
// launch, so the body runs at least once.
struct WhileGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    WhileGraph() = default;
    WhileGraph(const WhileGraph &) = delete;
    WhileGraph &operator=(const WhileGraph &) = delete;
    ~WhileGraph() { reset(); }
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    template <class Body>
    hc_status build(Body &&body, const char *who) {
        reset();
        HC_CUDA_TRY(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle cond;
        HC_CUDA_TRY(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = cond;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        HC_CUDA_TRY(cudaGraphAddNode(&node, graph, nullptr, 0, &np));
        // Captured on a private stream, so the caller's stream may be any kind.
        cudaStream_t cs;
        HC_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t e =
            cudaStreamBeginCaptureToGraph(cs, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            body(cs, cond);
            cudaGraph_t captured = nullptr;
            e = cudaStreamEndCapture(cs, &captured);
        }
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) return fail(HC_ERR_CUDA, "%s: epoch graph capture: %s", who, cudaGetErrorString(e));
        HC_CUDA_TRY(cudaGraphInstantiate(&exec, graph, 0));
        return HC_OK;
    }
};

}  // namespace hc
