// selftest.cu -- self-test of the bounded waits that every tensor-core kernel
// relies on to never hang the GPU.
//
// One CTA waits, with the same helper and time limit as the correlator
// kernels (tc_common.cuh: mbar_wait, kWaitLimitNs), on an mbarrier phase that
// nothing completes.  mode 0: the wait must give up when the time limit runs
// out.  mode 1: a second warp raises the CTA's abort flag after ~10 ms and the
// wait must give up at once.  mode 2: as mode 1, and the CTA then records the
// give-up in the error word of the allocation-free entry point, the way a
// correlator CTA records it in its launch's error word, so that
// chx_noalloc_check can be tested.  Either way the kernel records the outcome
// and the elapsed time and returns normally, so the context stays usable.
#include "tc_common.cuh"

namespace chx {
namespace {

using namespace tc;

__global__ void __launch_bounds__(64, 1) bounded_wait_selftest_kernel(int mode, int *result,
                                                                         int *err_word) {
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_word;
    volatile int *abort_flag = &abort_word;
    const uint32_t b = smem_u32(&bar);
    if (threadIdx.x == 0) {
        mbar_init(b, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint64_t t0 = globaltimer();
        // Phase 0 of a fresh barrier completes only after one arrival, and
        // nothing arrives.
        const bool completed = mbar_wait(b, 0, abort_flag);
        result[0] = completed ? 1 : 0;
        result[1] = (int)((globaltimer() - t0) / 1000000ull);
        if (!completed && mode == 2) atomicOr(err_word, 0x1000);
    } else if (threadIdx.x == 32 && mode >= 1) {
        const uint64_t t0 = globaltimer();
        while (globaltimer() - t0 < 10000000ull) {
        }
        *abort_flag = 1;
    }
}

}  // namespace
}  // namespace chx

using namespace chx;

extern "C" int chx_selftest_bounded_wait(int device, int mode, int *elapsed_ms) {
    clear_error();
    if (mode < 0 || mode > 2) return fail(CHX_E_INVALID, "mode=%d not in {0,1,2}", mode);
    int ndev = 0;
    CHX_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(CHX_E_INVALID, "device=%d", device);
    DeviceGuard g(device);
    int *err_word = nullptr;
    if (mode == 2) CHX_CUDA(noalloc_error_word(&err_word));
    int *d_result = nullptr;
    CHX_CUDA(cudaMalloc(&d_result, 2 * sizeof(int)));
    int h[2] = {-1, -1};
    cudaError_t e = cudaMemset(d_result, 0xff, 2 * sizeof(int));
    if (e == cudaSuccess) {
        bounded_wait_selftest_kernel<<<1, 64>>>(mode, d_result, err_word);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(h, d_result, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d_result);
    if (e != cudaSuccess) return cuda_fail(e, "bounded-wait self-test");
    if (elapsed_ms) *elapsed_ms = h[1];
    if (h[0] == 1) return fail(CHX_E_INVALID, "the wait completed although nothing arrived");
    return fail(CHX_E_TIMEOUT, "the bounded wait gave up after %d ms (mode %d)", h[1], mode);
}
