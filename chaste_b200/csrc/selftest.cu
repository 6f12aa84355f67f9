// Self-test of the bounded device waits (include/chaste_gpu.h,
// cg_selftest_barrier_timeout): a wait that nothing can satisfy must end by its
// time limit with kStatusBarrierTimeout, and the context must stay usable.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/chaste_gpu.h"
#include "kernels/common.cuh"

using namespace chb;

namespace {

// Every block arrives once, then waits for one arrival more than the grid has.
__global__ void selftest_wait_kernel(GridSync* gs, int* status, unsigned long long limit_ns,
                                     unsigned long long* waited_ns) {
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(gs->count);
        cnt.fetch_add(1u, cuda::memory_order_release);
        const unsigned long long t0 = global_ns();
        wait_count(&gs->count, gridDim.x + 1, status, limit_ns);
        const unsigned long long dt = global_ns() - t0;
        atomicMax(waited_ns, dt);
    }
    grid_exit(gs);
}

}  // namespace

extern "C" int cg_selftest_barrier_timeout(int device, double limit_ms, int* status_bits, double* waited_ms) {
    if (!status_bits || !(limit_ms >= 1.0 && limit_ms <= 2000.0)) return CG_ERR_ARG;
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) {
        cudaGetLastError();
        return CG_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return CG_ERR_CUDA;
    struct Scratch {
        GridSync gs;
        int status;
        int pad;
        unsigned long long waited;
    };
    Scratch* d = nullptr;
    if (cudaMalloc(&d, sizeof(Scratch)) != cudaSuccess) {
        cudaGetLastError();
        return CG_ERR_NOMEM;
    }
    int rc = CG_OK;
    Scratch h{};
    if (cudaMemset(d, 0, sizeof(Scratch)) != cudaSuccess) rc = CG_ERR_CUDA;
    if (rc == CG_OK) {
        selftest_wait_kernel<<<4, 32>>>(&d->gs, &d->status, (unsigned long long)(limit_ms * 1e6), &d->waited);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(&h, d, sizeof(Scratch), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = CG_ERR_CUDA;
    }
    cudaFree(d);
    if (rc != CG_OK) return rc;
    *status_bits = h.status;
    if (waited_ms) *waited_ms = (double)h.waited * 1e-6;
    return CG_OK;
}
