// cutlass_gemm_api.h -- drop-in C++ header for callers of the reference's HERK
// API, cutlass_interface/cutlass_gemm_api.h:157-789 (class
// cutlass_gemm_api::CutlassComplexGemm).  Same namespace, class name, enum
// names and ordinals, and herk / init_herk / end_herk / setter signatures, so
// that code written against the reference compiles unchanged and links
// against libftdx.so.  Every call forwards to the C ABI in ftdx.h.
//
// Differences a caller can observe:
//  * herk returns a non-zero ftdx_status instead of throwing for unsupported
//    combinations (compute precision FP6/FP4, which the reference maps to its
//    MX block-scaled GEMMs).
//  * K < 16 needs no padding by the caller (any K >= 1 is handled).
//  * set_direct_herk_graph(true) turns on graph capture and replay of whole
//    herk calls (ftdx_set_graph_mode), as the reference's direct-HERK graph
//    cache does (cutlass_gemm_api.cu:200-315); false releases the graphs.
//  * set_herk_mode picks this library's kernel: ForceDirect = the single-CTA
//    persistent tcgen05 kernel, ForceBaseline = the CTA-pair (cta_group::2)
//    kernel, Auto = the autotuner's choice.  While a mode is forced, herk
//    calls skip the strategy tuning, so the forced kernel runs.
//  * TileConfig, DirectTileConfig, PowerMode and GemmMode select tiles of the
//    reference's CUTLASS and mma.sync kernels, which this library does not
//    have; they are recorded and have no effect (the tcgen05 kernels' tiles
//    and pipeline depth are fixed; the autotuner picks their launch shape).
//  * The planar-complex GEMM / power-beamformer methods of the reference are
//    not part of this library.
#pragma once
#include <cuda_runtime.h>
#include <string>

#if defined(__GNUC__)
#define FTDX_SHIM_API __attribute__((visibility("default")))
#else
#define FTDX_SHIM_API
#endif

namespace cutlass_gemm_api {

enum class InputPrecision { FP16, INT4 };
enum class ComputePrecision { FP8, FP6, FP4 };
enum class OutputPrecision { FP16, FP32 };
enum class OutputFormat { PackedTriangle };
enum class HerkMode { Auto, ForceDirect, ForceBaseline };
enum class TileConfig {
  Auto, HerkOptimal, GemmOptimal, WideN, Cluster1x2, Cluster2x2, SmallTile, Pingpong, PingpongSmall
};
enum class PowerMode { Auto, ForceDirect, Force4M };
enum class DirectTileConfig { Auto, K32_B3, K64_B2, K64_B3, K128_B2 };
enum class GemmMode { Auto, ForceDirect, Force4M };

class FTDX_SHIM_API CutlassComplexGemm {
 public:
  CutlassComplexGemm();
  ~CutlassComplexGemm();

  // C = alpha * A * A^H + beta * C, packed lower triangle (see ftdx_herk).
  int herk(const void* A, void* C, int N, int K, int batch_count,
           InputPrecision input = InputPrecision::FP16,
           ComputePrecision compute = ComputePrecision::FP8,
           OutputPrecision output = OutputPrecision::FP16,
           OutputFormat format = OutputFormat::PackedTriangle, float alpha = 1.0f,
           float beta = 0.0f, cudaStream_t stream = nullptr, bool tune = true);

  void init_herk(int N, int K, int batch_count, cudaStream_t stream = nullptr);
  void end_herk();

  void set_tune_cache_path(const std::string& path);
  void set_strategy_tune_verbosity(int level);
  void set_gemm_tune_verbosity(int level);
  void set_gemm_tune_cache_path(const std::string& path);
  void set_kernel_tune_verbosity(int level);
  void set_kernel_tune_cache_path(const std::string& path);
  void set_herk_mode(HerkMode mode);
  void set_tile_config(TileConfig config);
  void set_direct_tile_config(DirectTileConfig config);
  void set_direct_herk_graph(bool enable);
  void set_power_mode(PowerMode mode);
  void set_gemm_mode(GemmMode mode);
  void set_auto_tune(bool enable);

  static void print_build_info();

  // Not in the reference: the underlying ftdx_handle (created on first use),
  // for callers that want this library's own C ABI on the same state.
  void* native_handle();

  CutlassComplexGemm(const CutlassComplexGemm&) = delete;
  CutlassComplexGemm& operator=(const CutlassComplexGemm&) = delete;

 private:
  struct Impl;
  Impl* impl_;
};

}  // namespace cutlass_gemm_api
