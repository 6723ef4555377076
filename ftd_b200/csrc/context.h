// context.h -- internal state behind an ftdx_handle, shared by the C-ABI
// translation units (ftdx_api.cu, herk_api.cu, ...).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <list>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/ftdx.h"
#include "herk_fp8.cuh"

namespace ftdx {

// Device-resident tile list + channel table for one problem shape.
struct Plan {
  TileDesc* d_tiles = nullptr;
  ChanDesc* d_chans = nullptr;
  int num_tiles = 0;
  int num_chans = 0;
  ~Plan();
};

constexpr int kStoreFp6 = 4;
constexpr int kStoreS8 = 8;   // with store mode 2: signed 8-bit operands, kind::i8 MMAs
constexpr int kStoreFused = 16;  // alone (mode 0 + 16): QC promotion fused into the single-CTA kernel
// Launch strategy of the correlator kernel; chosen by the autotuner.
struct Strategy {
  // 0: direct stores, 1: shared-memory staging + bulk copies,
  // 2: CTA-pair kernel (256 x 128 tiles on two SMs, direct stores);
  // 3: CTA-pair kernel with bulk-copy stores for interior tiles;
  // + kStoreFp6: operands as packed FP6 E3M2 planes (QC input, exact);
  // + kStoreS8 (pair only): signed 8-bit planes, integer MMAs (QC input, exact)
  // kStoreFused (alone): single CTA, direct stores, the QC bytes converted to
  // E4M3 inside the correlator (uniform INT4 calls; others run as 0)
  int store_mode = 0;
  int grid = 0;        // persistent CTAs (0: one per SM); -1: one CTA per tile (not persistent)
  int splits = 1;      // split-K: K is cut into this many ranges, partials summed afterwards
  bool operator==(const Strategy& o) const {
    return store_mode == o.store_mode && grid == o.grid && splits == o.splits;
  }
};

// Autotune cache key: device, problem shape and precisions.
struct TuneKey {
  std::string device;
  int n, kp, batch, input, output;
  bool operator<(const TuneKey& o) const {
    return std::tie(device, n, kp, batch, input, output) <
           std::tie(o.device, o.n, o.kp, o.batch, o.input, o.output);
  }
};
struct TuneEntry {
  Strategy st;
  float ms = 0.f;
};

// One captured launch sequence (promotion + correlator) for graph replay.
struct GraphKey {
  const void* a;
  void* c;
  int n, k, batch, input, output;
  float alpha, beta;
  int store_mode, grid, splits;
  bool operator==(const GraphKey& o) const {
    return a == o.a && c == o.c && n == o.n && k == o.k && batch == o.batch &&
           input == o.input && output == o.output && alpha == o.alpha && beta == o.beta &&
           store_mode == o.store_mode && grid == o.grid && splits == o.splits;
  }
};
struct GraphEntry {
  GraphKey key;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

}  // namespace ftdx

struct ftdx_context {
  int device = 0;
  int sm_count = 148;
  int pair_grid = -1;  // cached pair_grid_limit (-1: not queried yet)
  int verbosity = 0;
  std::string device_name;
  std::string last_error;
  // FP8 operand workspace (grown on demand, or pre-sized by ftdx_init_herk)
  uint8_t* z = nullptr;
  size_t z_cap = 0;
  // float inputs: promotion arrival words [32 x batch], amax[batch], qscale[batch], out_scale[batch]
  uint8_t* aux = nullptr;
  size_t aux_cap = 0;
  uint32_t* d_status = nullptr;
  // split-K partial triangles (grown on demand)
  uint8_t* split_ws = nullptr;
  size_t split_ws_cap = 0;
  // stridedBatchGEMM's FP16 staging (narrowed input, FP16 triangles), grown on demand
  uint8_t* strided_ws = nullptr;
  size_t strided_ws_cap = 0;
  int strided_mode = 0;  // FTDX_STRIDED_REFERENCE_FP16 or FTDX_STRIDED_SCALED_FP8
  std::map<std::tuple<int, int, int>, std::unique_ptr<ftdx::Plan>> plans;  // (N, kblocks, batch)
  std::map<uint64_t, std::shared_ptr<void>> vplans;  // batched-call plans by fingerprint
  // strategy of untuned calls (ftdx_set_strategy)
  ftdx::Strategy default_strategy;
  // autotuner
  std::string tune_cache;
  std::map<ftdx::TuneKey, ftdx::TuneEntry> tuned;
  int cache_bad_lines = 0;
  // graph replay (most recently used first)
  bool graph_mode = false;
  cudaStream_t capture_stream = nullptr;
  std::list<ftdx::GraphEntry> graphs;
  // kernel timing (ftdx_set_profiling)
  bool profiling = false;
  struct Timed {
    cudaEvent_t a, b;
    int kind;  // 0 = correlator, 1 = promotion
  };
  std::vector<Timed> timed;
  std::vector<cudaEvent_t> event_pool;
  // imaging workspace and FFT plans (imaging.cu), created on first use
  std::shared_ptr<void> imaging;
};

namespace ftdx {

constexpr size_t kGraphCacheSize = 4;

ftdx_status fail(ftdx_handle h, ftdx_status s, const char* fmt, ...);
ftdx_status cuda_fail(ftdx_handle h, cudaError_t e, const char* what);
bool stream_capturing(cudaStream_t s);
ftdx_status ensure_workspace(ftdx_handle h, size_t bytes, cudaStream_t s);
ftdx_status ensure_aux(ftdx_handle h, size_t bytes, cudaStream_t s);
// pair: tiles of the CTA-pair kernel (tj over 256 inputs, ti over 128);
// upper (pair only): the packed-upper XEngine format's tiles, tj over 256
// column inputs c and ti over 128 row inputs r <= c
ftdx_status get_plan(ftdx_handle h, int N, int kblocks, int batch, cudaStream_t s,
                     const Plan** out, bool pair = false, int splits = 1, bool upper = false);
ftdx_status ensure_split_ws(ftdx_handle h, size_t bytes, cudaStream_t s);
// fp6: planes of packed E3M2 codes (the kernels' fp6 operand form)
ftdx_status encode_planes_map(ftdx_handle h, uint8_t* z, int64_t rows, int64_t Kp,
                              CUtensorMap* tm, int box_rows = kTile, int nplanes = 2,
                              bool fp6 = false);
// 2-D map over raw QC bytes [rows][K] (K a multiple of 16, qc 16-byte
// aligned): 128-byte x 128-row boxes, unswizzled, zeros past K.
ftdx_status encode_qc_map(ftdx_handle h, const void* qc, int64_t rows, int K, CUtensorMap* tm);
// Even number of CTAs of the pair kernel that can be resident at once.
int pair_grid_limit(ftdx_handle h);
inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
void* tensor_map_encoder();  // cuTensorMapEncodeTiled through the runtime
// Text set by set_thread_error on the calling thread (empty: none).
const std::string& thread_error();

// Event pair around one kernel launch when profiling is on (never during capture).
struct ScopedTimer {
  ftdx_handle h;
  cudaStream_t s;
  int kind;
  cudaEvent_t a = nullptr;
  ScopedTimer(ftdx_handle h_, cudaStream_t s_, int kind_);
  ~ScopedTimer();
};

void release_graphs(ftdx_handle h);
void load_tune_cache(ftdx_handle h);

// Autotuning and graph replay shared by the correlator entry points.
using LaunchFn = std::function<ftdx_status(const Strategy&, cudaStream_t)>;
std::vector<Strategy> default_candidates(ftdx_handle h, bool fp32_out, bool pair_ok);
ftdx_status tune_sweep(ftdx_handle h, const LaunchFn& launch, const std::vector<Strategy>& cands,
                       cudaStream_t s, TuneEntry* best);
void record_tuned(ftdx_handle h, const TuneKey& k, const TuneEntry& e);
ftdx_status graph_launch(ftdx_handle h, const GraphKey& key,
                         const std::function<ftdx_status(cudaStream_t)>& launch, cudaStream_t s);

}  // namespace ftdx
