// cutlass_api_harness.cpp -- C entry points over the reference's own public
// HERK API, cutlass_gemm_api::CutlassComplexGemm
// (cutlass_interface/cutlass_gemm_api.h:157-789), which build_cutlass_ref.sh
// compiles unmodified from the reference's sources.  bench.py times the
// reference's GPU dispatch through them on the same QC input as this library:
// its default (HerkMode::Auto, K-adaptive), its direct kernel
// (ForceDirect) and its CUTLASS tcgen05 sub-GEMM baseline (ForceBaseline).
// The reference's autotuner is never run (tune = false), so its default tile
// configuration is used; exceptions become a -1 return.
#include <cuda_runtime.h>

#include "cutlass_gemm_api.h"

using cutlass_gemm_api::ComputePrecision;
using cutlass_gemm_api::CutlassComplexGemm;
using cutlass_gemm_api::HerkMode;
using cutlass_gemm_api::InputPrecision;
using cutlass_gemm_api::OutputFormat;
using cutlass_gemm_api::OutputPrecision;

extern "C" {

void* ref_api_create() {
  try {
    return new CutlassComplexGemm();
  } catch (...) {
    return nullptr;
  }
}

void ref_api_destroy(void* h) { delete static_cast<CutlassComplexGemm*>(h); }

// Tile configuration of the reference's CUTLASS baseline GEMMs
// (cutlass_gemm_api::TileConfig ordinal): only the single-CTA-cluster ones
// are accepted (0 Auto, 1 HerkOptimal 128x128, 2 GemmOptimal 128x128,
// 3 WideN 128x256, 6 SmallTile 128x64); -2 for any other.
int ref_api_set_tile_config(void* h, int cfg) {
  using cutlass_gemm_api::TileConfig;
  TileConfig tc;
  switch (cfg) {
    case 0: tc = TileConfig::Auto; break;
    case 1: tc = TileConfig::HerkOptimal; break;
    case 2: tc = TileConfig::GemmOptimal; break;
    case 3: tc = TileConfig::WideN; break;
    case 6: tc = TileConfig::SmallTile; break;
    default: return -2;
  }
  try {
    static_cast<CutlassComplexGemm*>(h)->set_tile_config(tc);
    return 0;
  } catch (...) {
    return -1;
  }
}

// Pre-allocates the reference's HERK buffers for up to (N, K, batch).
int ref_api_init_herk(void* h, int N, int K, int batch, void* stream) {
  try {
    static_cast<CutlassComplexGemm*>(h)->init_herk(N, K, batch,
                                                    static_cast<cudaStream_t>(stream));
    return 0;
  } catch (...) {
    return -1;
  }
}

// C = A A^H for QC int4 input A [batch][N][K], FP8 compute, FP32 packed lower
// triangles.  mode 0: HerkMode::Auto, 1: ForceDirect, 2: ForceBaseline.
int ref_api_herk_qc_fp32(void* h, const void* A, void* C, int N, int K, int batch, int mode,
                         void* stream) {
  try {
    auto* g = static_cast<CutlassComplexGemm*>(h);
    g->set_herk_mode(mode == 1   ? HerkMode::ForceDirect
                     : mode == 2 ? HerkMode::ForceBaseline
                                 : HerkMode::Auto);
    return g->herk(A, C, N, K, batch, InputPrecision::INT4, ComputePrecision::FP8,
                   OutputPrecision::FP32, OutputFormat::PackedTriangle, 1.f, 0.f,
                   static_cast<cudaStream_t>(stream), false);
  } catch (...) {
    return -1;
  }
}

// C = alpha A A^H + beta C through the reference's herk with its other input
// and output forms: input 0 = interleaved FP16 complex [batch][N][K][2],
// 1 = QC int4 bytes; output 0 = FP16, 1 = FP32 packed triangles; FP8 compute;
// mode as above.
int ref_api_herk(void* h, const void* A, void* C, int N, int K, int batch, int input, int output,
                 float alpha, float beta, int mode, void* stream) {
  try {
    auto* g = static_cast<CutlassComplexGemm*>(h);
    g->set_herk_mode(mode == 1   ? HerkMode::ForceDirect
                     : mode == 2 ? HerkMode::ForceBaseline
                                 : HerkMode::Auto);
    return g->herk(A, C, N, K, batch, input == 1 ? InputPrecision::INT4 : InputPrecision::FP16,
                   ComputePrecision::FP8, output == 1 ? OutputPrecision::FP32 : OutputPrecision::FP16,
                   OutputFormat::PackedTriangle, alpha, beta, static_cast<cudaStream_t>(stream),
                   false);
  } catch (...) {
    return -1;
  }
}

}  // extern "C"
