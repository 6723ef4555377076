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
//  * The CUTLASS-baseline tuning knobs (TileConfig, DirectTileConfig,
//    HerkMode, PowerMode, GemmMode) are accepted and recorded; this library
//    has one tcgen05 kernel family, whose launch shape the autotuner picks.
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

  CutlassComplexGemm(const CutlassComplexGemm&) = delete;
  CutlassComplexGemm& operator=(const CutlassComplexGemm&) = delete;

 private:
  struct Impl;
  Impl* impl_;
};

}  // namespace cutlass_gemm_api
