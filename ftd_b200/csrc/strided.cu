// strided.cu -- the HERK branch of quda::stridedBatchGEMMCutlass
// (lib/cutlass_interface.cu:316-381 of the reference), the XEngine's BLAS
// entry: C = A A^H for [batch][n][k] interleaved complex64 A, packed lower
// triangles of complex64 out.
//
// Default arithmetic (FTDX_STRIDED_REFERENCE_FP16), as the reference does it:
// every FP32 component is narrowed to FP16 (round to nearest), the HERK runs
// on FP16 input with the unscaled FP16 -> E4M3 conversion (round to nearest,
// saturating at 448) and FP32 accumulation, each result is rounded to FP16
// and then widened back to FP32.  FTDX_STRIDED_SCALED_FP8 (opt-in) runs the
// library's per-channel-scaled FP8 mode with FP32 output instead, which keeps
// inputs of any magnitude in range and results in FP32.
#include <cuda_fp16.h>

#include "context.h"

namespace ftdx {
namespace {

// One complex sample per element: (re, im) FP32 -> FP16, round to nearest.
__global__ void __launch_bounds__(256) narrow_to_half_kernel(const float2* __restrict__ in,
                                                             __half2* __restrict__ out, int64_t n) {
  for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < n;
       x += int64_t(gridDim.x) * blockDim.x) {
    const float2 v = __ldcs(in + x);
    out[x] = __floats2half2_rn(v.x, v.y);
  }
}

__global__ void __launch_bounds__(256) widen_from_half_kernel(const __half2* __restrict__ in,
                                                              float2* __restrict__ out,
                                                              int64_t n) {
  for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < n;
       x += int64_t(gridDim.x) * blockDim.x)
    __stcs(out + x, __half22float2(in[x]));
}

int grid_for(int64_t items, int sm_count) {
  int64_t b = (items + 255) / 256;
  if (b > int64_t(sm_count) * 16) b = int64_t(sm_count) * 16;
  return int(b < 1 ? 1 : b);
}

ftdx_status ensure_strided_ws(ftdx_handle h, size_t bytes, cudaStream_t s) {
  if (bytes <= h->strided_ws_cap) return FTDX_OK;
  if (stream_capturing(s))
    return fail(h, FTDX_ERR_CAPACITY, "strided_batch_gemm: staging needed while capturing");
  if (h->strided_ws) {
    cudaStreamSynchronize(s);
    cudaFree(h->strided_ws);
    h->strided_ws = nullptr;
    h->strided_ws_cap = 0;
  }
  cudaError_t e = cudaMalloc(&h->strided_ws, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, FTDX_ERR_ALLOC, "cudaMalloc(%zu) for strided_batch_gemm: %s", bytes,
                cudaGetErrorString(e));
  }
  h->strided_ws_cap = bytes;
  return FTDX_OK;
}

}  // namespace
}  // namespace ftdx

using namespace ftdx;

extern "C" {

ftdx_status ftdx_set_strided_mode(ftdx_handle h, int mode) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (mode != FTDX_STRIDED_REFERENCE_FP16 && mode != FTDX_STRIDED_SCALED_FP8)
    return fail(h, FTDX_ERR_INVALID_ARG, "set_strided_mode: unknown mode %d", mode);
  h->strided_mode = mode;
  return FTDX_OK;
}

long long ftdx_strided_batch_gemm(ftdx_handle h, const void* A, const void* B, void* C, int m,
                                  int n, int k, int trans_a, int trans_b, int batch, int data_type,
                                  void* stream) {
  if (!h) return -1;
  constexpr int kOpN = 0, kOpC = 2, kComplexFloat = 2;
  const bool herk = A == B && trans_a == kOpC && trans_b == kOpN && m == n;
  if (!herk || data_type != kComplexFloat) {
    fail(h, FTDX_ERR_UNSUPPORTED,
         "strided_batch_gemm: only the HERK pattern (A == B, op(A) = A^H, op(B) = B, m == n, "
         "single complex) is implemented (got trans %d/%d, m %d, n %d, type %d)",
         trans_a, trans_b, m, n, data_type);
    return -1;
  }
  if (!A || !C || n < 1 || k < 1 || batch < 1) {
    fail(h, FTDX_ERR_INVALID_ARG, "strided_batch_gemm: null pointer or size < 1");
    return -1;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (h->strided_mode == FTDX_STRIDED_SCALED_FP8) {
    if (ftdx_herk(h, A, C, n, k, batch, FTDX_IN_FP32, FTDX_COMPUTE_FP8, FTDX_OUT_FP32,
                  FTDX_FORMAT_PACKED_TRIANGLE, 1.f, 0.f, stream, 1) != FTDX_OK)
      return -1;
  } else {
    if ((reinterpret_cast<uintptr_t>(A) & 7) != 0 || (reinterpret_cast<uintptr_t>(C) & 7) != 0) {
      fail(h, FTDX_ERR_INVALID_ARG, "strided_batch_gemm: A and C must be 8-byte aligned");
      return -1;
    }
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) {
      cuda_fail(h, e, "cudaSetDevice");
      return -1;
    }
    // staging: the narrowed input [batch][n][k] __half2, then the FP16 triangles
    const int64_t in_elems = int64_t(batch) * n * k;  // complex samples
    const int64_t P = int64_t(n) * (n + 1) / 2;
    const size_t in_bytes = size_t(round_up(in_elems * 4, 256));
    const size_t out_bytes = size_t(int64_t(batch) * P * 4);
    if (ensure_strided_ws(h, in_bytes + out_bytes, s) != FTDX_OK) return -1;
    uint8_t* a16 = h->strided_ws;
    uint8_t* c16 = h->strided_ws + in_bytes;
    narrow_to_half_kernel<<<grid_for(in_elems, h->sm_count), 256, 0, s>>>(
        static_cast<const float2*>(A), reinterpret_cast<__half2*>(a16), in_elems);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      cuda_fail(h, e, "strided_batch_gemm narrowing");
      return -1;
    }
    if (ftdx_herk(h, a16, c16, n, k, batch, FTDX_IN_FP16, FTDX_COMPUTE_FP8, FTDX_OUT_FP16,
                  FTDX_FORMAT_PACKED_TRIANGLE, 1.f, 0.f, stream, 1) != FTDX_OK)
      return -1;
    widen_from_half_kernel<<<grid_for(int64_t(batch) * P, h->sm_count), 256, 0, s>>>(
        reinterpret_cast<const __half2*>(c16), static_cast<float2*>(C), int64_t(batch) * P);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      cuda_fail(h, e, "strided_batch_gemm widening");
      return -1;
    }
  }
  uint32_t bits = 0;
  if (ftdx_device_status(h, stream, &bits) != FTDX_OK) return -1;
  return 8LL * m * n * k * batch;
}

}  // extern "C"
