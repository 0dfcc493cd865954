// Device-side time limits and the barrier self-check.
//
// Every bounded wait in this library (the grid barrier, the run limit of the
// persistent kernels, the epoch-loop limit of the batched paths) reads its
// bound from a __constant__ copy in its own translation unit.
// hc_set_time_limits writes all copies on one device, so that a test can make
// each wait run out in a millisecond and check that the call returns
// HC_ERR_TIMEOUT and leaves the handle usable.  hc_selftest_grid_barrier runs
// the grid barrier alone with one block held back: the others give up after
// the wait limit, record HC_ERR_TIMEOUT and return.
#include <mutex>
#include <vector>

#include "hc_device.cuh"

namespace hc {

namespace {
std::vector<LimitSetter> &limit_setters() {
    static std::vector<LimitSetter> v;
    return v;
}
std::mutex &limit_mutex() {
    static std::mutex m;
    return m;
}

__global__ void barrier_selftest(GridSync *gs, int withhold) {
    if ((int)blockIdx.x == withhold) return;  // this block never arrives
    grid_barrier(gs);
}
}  // namespace

void register_limit_setter(LimitSetter f) {
    std::lock_guard<std::mutex> lk(limit_mutex());
    limit_setters().push_back(f);
}

}  // namespace hc

using namespace hc;

extern "C" hc_status hc_set_time_limits(int32_t device, uint64_t wait_ns, uint64_t run_ns, uint64_t loop_ns) {
    clear_error();
    int prev = 0;
    HC_CUDA_TRY(cudaGetDevice(&prev));
    HC_CUDA_TRY(cudaSetDevice(device));
    TimeLimits t{wait_ns ? wait_ns : kWaitLimitNs, run_ns ? run_ns : kRunLimitNs, loop_ns ? loop_ns : kLoopLimitNs};
    hc_status st = HC_OK;
    {
        std::lock_guard<std::mutex> lk(limit_mutex());
        for (LimitSetter f : limit_setters())
            if ((st = f(t)) != HC_OK) break;
    }
    cudaSetDevice(prev);
    return st;
}

extern "C" hc_status hc_selftest_grid_barrier(int32_t device, int32_t blocks, int32_t withhold_block,
                                              int32_t *status_out) {
    clear_error();
    if (!status_out || blocks < 1 || blocks > 64 || withhold_block >= blocks)
        return fail(HC_ERR_INVALID_ARG, "hc_selftest_grid_barrier: bad arguments");
    int prev = 0;
    HC_CUDA_TRY(cudaGetDevice(&prev));
    HC_CUDA_TRY(cudaSetDevice(device));
    GridSync *gs = nullptr;
    HC_CUDA_TRY(cudaMalloc(&gs, sizeof(GridSync)));
    hc_status st = HC_OK;
    cudaError_t e = cudaMemset(gs, 0, sizeof(GridSync));
    if (e == cudaSuccess) {
        int w = withhold_block;
        void *params[] = {&gs, &w};
        count_launch();
        // A cooperative launch keeps every block resident, so the blocks that
        // wait cannot starve the one that arrives late.
        e = cudaLaunchCooperativeKernel((void *)barrier_selftest, dim3(blocks), dim3(32), params, 0, nullptr);
    }
    GridSync h{};
    if (e == cudaSuccess) e = cudaMemcpy(&h, gs, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(HC_ERR_CUDA, "hc_selftest_grid_barrier: %s", cudaGetErrorString(e));
    cudaFree(gs);
    cudaSetDevice(prev);
    if (st == HC_OK) *status_out = h.err;
    return st;
}
