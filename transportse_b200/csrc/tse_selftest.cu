// Self-test of the bounded waits every persistent kernel of the library
// relies on.  Each case runs one wait whose condition nothing ever makes true
// -- a grid barrier that counts one block more than the launch has, a
// counter barrier with an unreachable target, an mbarrier no one arrives at
// -- and records whether the wait gave up after its time limit and raised its
// error flag, as it must for a solver kernel to return
// TSE_STATUS_BARRIER_TIMEOUT instead of holding the GPU.  Nothing faults: the
// kernels only wait, give up and return.
#include "tse_dc.cuh"

namespace tse {

// result[which]: 1 = the wait returned false with its error flag raised
__global__ void __launch_bounds__(128) selftest_wait_kernel(int which, GridBarrier* bar,
                                                            unsigned* counter, int* result,
                                                            unsigned long long timeout_ns) {
    if (which == 0) {
        const bool ok = grid_sync(bar, gridDim.x + 1, timeout_ns);
        if (blockIdx.x == 0 && threadIdx.x == 0)
            result[0] = (!ok && *(volatile int*)&bar->error) ? 1 : 0;
    } else if (which == 1) {
        const bool ok = count_sync(counter, gridDim.x + 1, bar, timeout_ns);
        if (blockIdx.x == 0 && threadIdx.x == 0)
            result[1] = (!ok && *(volatile int*)&bar->error) ? 1 : 0;
    } else {
        __shared__ __align__(8) uint64_t mb;
        __shared__ int err;
        if (threadIdx.x == 0) {
            mbar_init(&mb, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            err = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const bool ok = mbar_wait_flag(&mb, 0u, (volatile int*)&err, timeout_ns);
            // complete the phase no one completed, so the barrier is left idle
            mbar_arrive(&mb);
            result[2] = (!ok && err) ? 1 : 0;
        }
        __syncthreads();
    }
}

}  // namespace tse

using namespace tse;

extern "C" int32_t tse_selftest_bounded_waits(int32_t* d_result, double timeout_s, void* d_ws,
                                              size_t ws_bytes, void* stream_) {
    if (!d_result || !d_ws || ws_bytes < 512 || !(timeout_s > 0.0)) return TSE_ERR_ARG;
    if (timeout_s > 5.0) timeout_s = 5.0;
    const unsigned long long ns = (unsigned long long)(timeout_s * 1e9);
    cudaStream_t stream = (cudaStream_t)stream_;
    GridBarrier* bar = (GridBarrier*)d_ws;
    unsigned* counter = (unsigned*)((char*)d_ws + 256);
    int* result = (int*)d_result;
    if (cudaMemsetAsync(d_result, 0, 3 * sizeof(int32_t), stream) != cudaSuccess) return TSE_ERR_LAUNCH;
    for (int which = 0; which < 3; ++which) {
        if (cudaMemsetAsync(d_ws, 0, 512, stream) != cudaSuccess) return TSE_ERR_LAUNCH;
        // the two blocks of the barrier cases wait on each other: co-resident
        // by a cooperative launch
        int w = which;
        void* args[] = {(void*)&w, (void*)&bar, (void*)&counter, (void*)&result, (void*)&ns};
        const cudaError_t e =
            which < 2 ? cudaLaunchCooperativeKernel((const void*)selftest_wait_kernel, dim3(2), dim3(128),
                                                    args, 0, stream)
                      : cudaLaunchKernel((const void*)selftest_wait_kernel, dim3(1), dim3(128), args, 0,
                                         stream);
        if (e != cudaSuccess) return TSE_ERR_LAUNCH;
    }
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}
