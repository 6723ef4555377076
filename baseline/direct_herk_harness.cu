// direct_herk_harness.cu -- C entry point around the reference's own direct
// HERK kernel and INT4 -> FP8 cast (extracted from the reference tree into
// baseline/_ref/ by build_direct_ref.sh, never committed), so that the
// benchmark can time the reference's Blackwell kernel on the same GPU, input
// and output layout as this library:
//   QC int4 [batch][N][K] bytes -> cast_int4_to_fp8_interleaved (interleaved
//   [re, im] E4M3, cutlass_gemm_api.cu:1566-1623) -> launch_herk_direct_fp8_precast
//   (herk_kernel_common.hpp:431-461, FP32 packed lower triangles, alpha 1, beta 0).
// The extracted text expects, from the reference's CUTLASS build,
// cutlass::Status, FillMode and CUDA_CHECK; minimal stand-ins follow.
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace cutlass {
enum class Status { kSuccess = 0, kErrorNotSupported = 1 };
}

namespace ref_direct {
enum class FillMode { Lower, Upper };
#define CUDA_CHECK(call) (void)(call)
#include "ref_direct_herk.inc"
#include "ref_qc_cast.inc"
#undef CUDA_CHECK
}  // namespace ref_direct

extern "C" {

// Bytes of FP8 staging the reference's path needs (2 per complex sample).
size_t ref_direct_herk_staging_bytes(int N, int K, int batch) {
  return size_t(2) * size_t(N) * size_t(K) * size_t(batch);
}

// qc: device, 16-byte aligned; fp8: device staging of the size above; C: device
// packed lower triangles [batch][N(N+1)/2] complex64.  0 on success, else the
// CUDA error (or -1 when the reference's launcher refuses).
int ref_direct_herk_qc(const uint8_t* qc, void* fp8, float* C, int N, int K, int batch,
                       cudaStream_t stream) {
  ref_direct::cast_int4_to_fp8_interleaved(qc, static_cast<__nv_fp8_e4m3*>(fp8),
                                           int64_t(N) * K * batch, stream);
  const auto st = ref_direct::launch_herk_direct_fp8_precast<float>(
      static_cast<const __nv_fp8_e4m3*>(fp8), C, N, K, batch, 1.0f, 0.0f,
      ref_direct::FillMode::Lower, stream);
  if (st != cutlass::Status::kSuccess) return -1;
  return int(cudaGetLastError());
}

}  // extern "C"
