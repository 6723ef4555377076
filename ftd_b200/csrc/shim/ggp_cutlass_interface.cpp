// ggp_cutlass_interface.cpp -- the GGP engine-boundary functions of
// lib/cutlass_interface.cu:150-381: namespace ggp over one process-wide
// CutlassComplexGemm, as the reference keeps one (:38-41), and
// quda::stridedBatchGEMMCutlass.  The ggp:: declarations are the ones
// callers forward-declare (lib/visibility_pipeline.cu:11-22,
// lib/visibility_bf.cpp:15-21).  Returns 0 on success, never exits.
#include <cuda_runtime.h>

#include "cutlass_gemm_api.h"
#include "ftdx.h"
#include "ggp_blas_interface.h"

using cutlass_gemm_api::ComputePrecision;
using cutlass_gemm_api::CutlassComplexGemm;
using cutlass_gemm_api::InputPrecision;
using cutlass_gemm_api::OutputFormat;
using cutlass_gemm_api::OutputPrecision;

namespace {
CutlassComplexGemm& api() {
  static CutlassComplexGemm instance;
  return instance;
}
bool g_herk_tune = false;
}  // namespace

namespace ggp {

FTDX_SHIM_API void initCutlassApi(int kernel_tune_verbosity, const char* kernel_tune_cache_path,
                                  const char* strategy_tune_cache_path, bool herk_tune,
                                  int strategy_tune_verbosity) {
  auto& a = api();
  if (kernel_tune_verbosity > 0) a.set_kernel_tune_verbosity(kernel_tune_verbosity);
  a.set_strategy_tune_verbosity(strategy_tune_verbosity);
  if (kernel_tune_cache_path) a.set_kernel_tune_cache_path(kernel_tune_cache_path);
  if (strategy_tune_cache_path) a.set_tune_cache_path(strategy_tune_cache_path);
  g_herk_tune = herk_tune;
}

// QC int4 [batch][N][K] -> FP32 packed lower triangles.
FTDX_SHIM_API int herkBatchedCutlassQC(const void* qc_data, void* tri_output, int N, int K,
                                       int batch, cudaStream_t stream) {
  return api().herk(qc_data, tri_output, N, K, batch, InputPrecision::INT4,
                    ComputePrecision::FP8, OutputPrecision::FP32, OutputFormat::PackedTriangle,
                    1.0f, 0.0f, stream, g_herk_tune);
}

// QC int4 -> FP16 packed lower triangles (overflows for K beyond ~668 with
// full-scale input, as in the reference).
FTDX_SHIM_API int herkBatchedCutlassQC_FP16(const void* qc_data, void* tri_output, int N, int K,
                                            int batch, cudaStream_t stream) {
  return api().herk(qc_data, tri_output, N, K, batch, InputPrecision::INT4,
                    ComputePrecision::FP8, OutputPrecision::FP16, OutputFormat::PackedTriangle,
                    1.0f, 0.0f, stream, g_herk_tune);
}

// Interleaved FP16 complex [batch][N][K][2] -> FP16 packed lower triangles.
FTDX_SHIM_API int herkBatchedCutlassFP16(const void* fp16_data, void* tri_output, int N, int K,
                                         int batch, cudaStream_t stream) {
  return api().herk(fp16_data, tri_output, N, K, batch, InputPrecision::FP16,
                    ComputePrecision::FP8, OutputPrecision::FP16, OutputFormat::PackedTriangle,
                    1.0f, 0.0f, stream, g_herk_tune);
}

}  // namespace ggp

namespace quda {

// The reference keeps this path on its process-wide CutlassComplexGemm; the
// HERK-detecting BLAS entry needs this library's strided call, so it has its
// own process-wide handle on the device current at the first call.
long long stridedBatchGEMMCutlass(void* A_data, void* B_data, void* C_data, QudaBLASParam param,
                                  QudaFieldLocation /*location*/) {
  static ftdx_handle h = nullptr;
  static ftdx_status created = [] {
    ftdx_config cfg{};
    cfg.device = -1;
    return ftdx_create(&h, &cfg);
  }();
  if (created != FTDX_OK) return -1;
  return ftdx_strided_batch_gemm(h, A_data, B_data, C_data, param.m, param.n, param.k,
                                 int(param.trans_a), int(param.trans_b), param.batch_count,
                                 int(param.data_type), nullptr);
}

}  // namespace quda
