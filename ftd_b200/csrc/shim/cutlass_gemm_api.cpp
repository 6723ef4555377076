// cutlass_gemm_api.cpp -- CutlassComplexGemm over the C ABI (ftdx.h).
// Mirrors cutlass_interface/cutlass_gemm_api.cu:1707-1878 (herk) and
// :1291-1353 (init_herk / end_herk) of the reference.
#include "cutlass_gemm_api.h"

#include <cstdio>
#include <cstdlib>

#include "ftdx.h"

namespace cutlass_gemm_api {

struct CutlassComplexGemm::Impl {
  ftdx_handle h = nullptr;
  ftdx_status create_status = FTDX_OK;
  bool auto_tune = false;
  bool direct_graph = false;
  int strategy_verbosity = 1;
  HerkMode herk_mode = HerkMode::Auto;
  TileConfig tile = TileConfig::Auto;
  DirectTileConfig direct_tile = DirectTileConfig::Auto;
  PowerMode power = PowerMode::Auto;
  GemmMode gemm = GemmMode::Auto;
  std::string tune_cache;

  ftdx_handle get() {
    if (!h && create_status == FTDX_OK) {
      ftdx_config cfg{};
      cfg.device = -1;
      cfg.verbosity = strategy_verbosity > 1 ? strategy_verbosity : 0;
      cfg.tune_cache = tune_cache.empty() ? nullptr : tune_cache.c_str();
      create_status = ftdx_create(&h, &cfg);
      if (create_status != FTDX_OK) {
        h = nullptr;
      } else {
        if (direct_graph) ftdx_set_graph_mode(h, 1);
        apply_mode();
      }
    }
    return h;
  }

  // HerkMode -> this library's kernel (store mode of ftdx_set_strategy)
  void apply_mode() {
    if (!h) return;
    switch (herk_mode) {
      case HerkMode::ForceBaseline:
        if (ftdx_set_strategy(h, 2, 0) != FTDX_OK) ftdx_set_strategy(h, 0, 0);
        break;
      case HerkMode::ForceDirect:
      case HerkMode::Auto: ftdx_set_strategy(h, 0, 0); break;
    }
  }
};

CutlassComplexGemm::CutlassComplexGemm() : impl_(new Impl()) {}

CutlassComplexGemm::~CutlassComplexGemm() {
  if (impl_->h) ftdx_destroy(impl_->h);
  delete impl_;
}

int CutlassComplexGemm::herk(const void* A, void* C, int N, int K, int batch_count,
                             InputPrecision input, ComputePrecision compute,
                             OutputPrecision output, OutputFormat format, float alpha, float beta,
                             cudaStream_t stream, bool tune) {
  ftdx_handle h = impl_->get();
  if (!h) return int(impl_->create_status);
  return int(ftdx_herk(h, A, C, N, K, batch_count, ftdx_input(int(input)),
                       ftdx_compute(int(compute)), ftdx_output(int(output)),
                       ftdx_format(int(format)), alpha, beta, static_cast<void*>(stream),
                       ((tune || impl_->auto_tune) && impl_->herk_mode == HerkMode::Auto) ? 1
                                                                                         : 0));
}

void CutlassComplexGemm::init_herk(int N, int K, int batch_count, cudaStream_t stream) {
  if (ftdx_handle h = impl_->get()) ftdx_init_herk(h, N, K, batch_count, stream);
}

void CutlassComplexGemm::end_herk() {
  if (impl_->h) ftdx_end_herk(impl_->h);
}

void CutlassComplexGemm::set_tune_cache_path(const std::string& path) {
  impl_->tune_cache = path;
  if (impl_->h) ftdx_set_tune_cache(impl_->h, path.c_str());
}
void CutlassComplexGemm::set_strategy_tune_verbosity(int level) {
  impl_->strategy_verbosity = level;
}
void CutlassComplexGemm::set_gemm_tune_verbosity(int) {}
void CutlassComplexGemm::set_gemm_tune_cache_path(const std::string&) {}
void CutlassComplexGemm::set_kernel_tune_verbosity(int) {}
void CutlassComplexGemm::set_kernel_tune_cache_path(const std::string&) {}
void CutlassComplexGemm::set_herk_mode(HerkMode mode) {
  impl_->herk_mode = mode;
  impl_->apply_mode();
}
void CutlassComplexGemm::set_tile_config(TileConfig config) { impl_->tile = config; }
void CutlassComplexGemm::set_direct_tile_config(DirectTileConfig config) {
  impl_->direct_tile = config;
}
void CutlassComplexGemm::set_direct_herk_graph(bool enable) {
  impl_->direct_graph = enable;
  if (impl_->h) ftdx_set_graph_mode(impl_->h, enable ? 1 : 0);
}
void CutlassComplexGemm::set_power_mode(PowerMode mode) { impl_->power = mode; }
void CutlassComplexGemm::set_gemm_mode(GemmMode mode) { impl_->gemm = mode; }
void CutlassComplexGemm::set_auto_tune(bool enable) { impl_->auto_tune = enable; }

void* CutlassComplexGemm::native_handle() { return static_cast<void*>(impl_->get()); }

void CutlassComplexGemm::print_build_info() {
  const int v = ftdx_version();
  std::printf("ftdx %d.%d: tcgen05 FP8 correlator for sm_100a\n", v >> 16, v & 0xffff);
  int dev = 0;
  cudaDeviceProp prop{};
  if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
    std::printf("  device %d: %s, sm_%d%d, %d SMs\n", dev, prop.name, prop.major, prop.minor,
                prop.multiProcessorCount);
}

}  // namespace cutlass_gemm_api
