// Self-test of the bounded waits every pipelined kernel here relies on.
//
// swe_selftest_wait_timeout launches one block that waits on an mbarrier
// which nothing ever arrives on, with the time-bounded sleeping wait of the
// pipelined stage kernels (tc::mbar_wait_timed).  The wait must give up after
// about limit_ns, write a status word and let the kernel return, so that the
// context stays usable and the host reads SWE_ERR_TIMEOUT.  It checks the
// timeout path without a fault, a trap or an unbounded loop.
#include <cuda_runtime.h>

#include "common.cuh"
#include "tcgen05.cuh"

namespace swe {
namespace {

__global__ void never_arrives_kernel(unsigned long long limit_ns, int* status, unsigned long long* waited_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    const uint64_t t0 = tc::globaltimer_ns();
    const bool ok = tc::mbar_wait_timed(&bar, 0, limit_ns, 1000);
    __syncthreads();
    if (threadIdx.x == 0) {
        *status = ok ? 0 : 1;
        *waited_ns = tc::globaltimer_ns() - t0;
    }
}

}  // namespace
}  // namespace swe

extern "C" int swe_selftest_wait_timeout(double limit_s, double* waited_s) {
    using namespace swe;
    if (!(limit_s > 0.0) || limit_s > 2.0) {
        set_error("swe_selftest_wait_timeout: limit must be in (0, 2] seconds");
        return SWE_ERR_ARG;
    }
    int* status = nullptr;
    unsigned long long* waited = nullptr;
    SWE_CUDA_TRY(cudaMalloc(&status, sizeof(int)));
    SWE_CUDA_TRY(cudaMalloc(&waited, sizeof(unsigned long long)));
    never_arrives_kernel<<<1, 32>>>((unsigned long long)(limit_s * 1e9), status, waited);
    count_launch();
    int h = -1;
    unsigned long long w = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&w, waited, sizeof(w), cudaMemcpyDeviceToHost);
    cudaFree(status);
    cudaFree(waited);
    if (e != cudaSuccess) {
        set_error("swe_selftest_wait_timeout: %s", cudaGetErrorString(e));
        return SWE_ERR_CUDA;
    }
    if (waited_s) *waited_s = (double)w * 1e-9;
    if (h == 1) {
        set_error("bounded wait gave up after %.3f s (as intended)", (double)w * 1e-9);
        return SWE_ERR_TIMEOUT;
    }
    set_error("swe_selftest_wait_timeout: the wait completed although nothing arrived");
    return SWE_ERR_STATE;
}
