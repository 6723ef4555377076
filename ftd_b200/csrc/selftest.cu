// selftest.cu -- exercises the failure path of the kernels' bounded waits
// without faulting anything (ftdx_wait_selftest): one CTA waits, with a short
// limit, on an mbarrier that nothing arrives on, then on a global flag that
// nothing sets (the wait between the blocks of the cooperative FP8
// promotion); when both give up it records the timeout in the handle's
// status word and returns.  The context stays usable.
#include "context.h"
#include "sm100.cuh"

namespace ftdx {
namespace {

__device__ uint32_t g_never_set = 0;  // no code writes it

__global__ void wait_selftest_kernel(uint32_t* status, uint64_t limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    dev::mbar_init(dev::smem_u32(&bar), 1);  // one arrival expected; none comes
    abort_flag = 0;
    dev::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int* ab = &abort_flag;
    const bool bar_done = dev::mbar_wait_limit(dev::smem_u32(&bar), 0, ab, limit_ns);
    const bool flag_done = dev::flag_wait_limit(&g_never_set, 1u, limit_ns);
    if (!bar_done && !flag_done) atomicOr(status, dev::kStatusTimeoutOther);
  }
}

}  // namespace
}  // namespace ftdx

using namespace ftdx;

extern "C" ftdx_status ftdx_wait_selftest(ftdx_handle h, int timeout_ms, void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (timeout_ms < 1 || timeout_ms > 2000)
    return fail(h, FTDX_ERR_INVALID_ARG, "wait_selftest: timeout_ms must be 1..2000");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  wait_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(
      h->d_status, uint64_t(timeout_ms) * 1000000ull);
  e = cudaGetLastError();
  return e == cudaSuccess ? FTDX_OK : cuda_fail(h, e, "wait selftest launch");
}
