// ftdx_api.cu -- C ABI core: handles, workspace, tile plans, tensor maps,
// device status and kernel timing.  The correlator entry points are in
// herk_api.cu.  See include/ftdx.h.
#include <cudaTypedefs.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <algorithm>
#include <mutex>
#include <set>
#include <utility>

#include "context.h"

namespace ftdx {

Plan::~Plan() {
  if (d_tiles) cudaFree(d_tiles);
  if (d_chans) cudaFree(d_chans);
}

static PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

static std::string& thread_error_text() {
  thread_local std::string t;  // last failure of a handle-less call on this thread
  return t;
}
const std::string& thread_error() { return thread_error_text(); }

void set_thread_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  thread_error_text() = buf;
}

cudaError_t ensure_smem_limit(const void* kernel, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({dev, kernel})) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  if (e == cudaSuccess) done.insert({dev, kernel});
  return e;
}

void* tensor_map_encoder() { return reinterpret_cast<void*>(get_encode_fn()); }

ftdx_status fail(ftdx_handle h, ftdx_status s, const char* fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    h->last_error = buf;
    if (h->verbosity > 0) fprintf(stderr, "ftdx: %s\n", buf);
  }
  return s;
}

ftdx_status cuda_fail(ftdx_handle h, cudaError_t e, const char* what) {
  return fail(h, FTDX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

bool stream_capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return st != cudaStreamCaptureStatusNone;
}

ftdx_status ensure_workspace(ftdx_handle h, size_t bytes, cudaStream_t s) {
  if (bytes <= h->z_cap) return FTDX_OK;
  if (stream_capturing(s))
    return fail(h, FTDX_ERR_CAPACITY,
                "workspace of %zu bytes needed while capturing (have %zu); call ftdx_init_herk "
                "first",
                bytes, h->z_cap);
  if (h->z) {
    cudaDeviceSynchronize();  // every queued user of the old buffer is done
    cudaFree(h->z);
    h->z = nullptr;
    h->z_cap = 0;
    release_graphs(h);  // captured graphs point at the old buffer
  }
  cudaError_t e = cudaMalloc(&h->z, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, FTDX_ERR_ALLOC, "cudaMalloc(%zu) for the FP8 operand: %s", bytes,
                cudaGetErrorString(e));
  }
  h->z_cap = bytes;
  return FTDX_OK;
}

ftdx_status ensure_split_ws(ftdx_handle h, size_t bytes, cudaStream_t s) {
  if (bytes <= h->split_ws_cap) return FTDX_OK;
  if (stream_capturing(s))
    return fail(h, FTDX_ERR_CAPACITY, "split-K workspace needed while capturing; call once first");
  if (h->split_ws) {
    cudaDeviceSynchronize();
    cudaFree(h->split_ws);
    h->split_ws = nullptr;
    h->split_ws_cap = 0;
    release_graphs(h);
  }
  cudaError_t e = cudaMalloc(&h->split_ws, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, FTDX_ERR_ALLOC, "cudaMalloc(%zu) for split-K partials: %s", bytes,
                cudaGetErrorString(e));
  }
  h->split_ws_cap = bytes;
  return FTDX_OK;
}

ftdx_status ensure_aux(ftdx_handle h, size_t bytes, cudaStream_t s) {
  if (bytes <= h->aux_cap) return FTDX_OK;
  if (stream_capturing(s))
    return fail(h, FTDX_ERR_CAPACITY, "scale buffer needed while capturing; call once first");
  if (h->aux) {
    cudaDeviceSynchronize();
    cudaFree(h->aux);
    h->aux = nullptr;
    h->aux_cap = 0;
    release_graphs(h);
  }
  cudaError_t e = cudaMalloc(&h->aux, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, FTDX_ERR_ALLOC, "cudaMalloc(%zu) for channel scales: %s", bytes,
                cudaGetErrorString(e));
  }
  h->aux_cap = bytes;
  return FTDX_OK;
}

// Lower-triangle tile list for `batch` channels of N inputs, channel-major so
// that concurrently running CTAs share a channel's operand in L2.
ftdx_status get_plan(ftdx_handle h, int N, int kblocks, int batch, cudaStream_t s,
                     const Plan** out, bool pair, int splits, bool upper) {
  upper = upper && pair;
  // kblocks < 2^23 (K <= 2^30) and splits <= 32, so pair, split-K and
  // upper-format pair plans never share a key with others
  auto key = std::make_tuple(N, kblocks + (pair ? (1 << 24) : 0) + ((splits - 1) << 25) +
                                    (upper ? (1 << 30) : 0),
                             batch);
  auto it = h->plans.find(key);
  if (it != h->plans.end()) {
    *out = it->second.get();
    return FTDX_OK;
  }
  if (stream_capturing(s))
    return fail(h, FTDX_ERR_CAPACITY,
                "tile plan for N=%d batch=%d built while capturing; call ftdx_init_herk first", N,
                batch);
  const int nb = (N + kTile - 1) / kTile;
  // split-K: channel entry c*splits + s covers k-blocks [kb0, kb0 + kblocks) of
  // channel c and writes partial triangle c*splits + s
  std::vector<ChanDesc> chans(size_t(batch) * splits);
  std::vector<TileDesc> tiles;
  tiles.reserve(size_t(batch) * splits * nb * (nb + 1) / 2);
  for (int c = 0; c < batch; ++c) {
    for (int sp = 0; sp < splits; ++sp) {
      const int vc = c * splits + sp;
      const int kb_lo = int(int64_t(sp) * kblocks / splits);
      const int kb_hi = int(int64_t(sp + 1) * kblocks / splits);
      chans[vc].n = N;
      chans[vc].kblocks = kb_hi - kb_lo;
      chans[vc].kb0 = kb_lo;
      chans[vc].row0 = int64_t(c) * N;
      chans[vc].out0 = int64_t(vc) * (int64_t(N) * (N + 1) / 2);
      chans[vc].out_ptr = 0;
      if (upper) {
        // packed-upper pair tiles: tj over 256 column inputs c (the TMEM
        // lanes), ti over 128 row inputs r <= c (the TMEM columns)
        for (int tj = 0; tj < (N + 255) / 256; ++tj)
          for (int ti = 0; ti < nb && ti <= 2 * tj + 1; ++ti)
            tiles.push_back(TileDesc{vc, uint16_t(ti), uint16_t(tj)});
        continue;
      }
      for (int ti = 0; ti < nb; ++ti)
        for (int tj = 0; tj <= (pair ? ti / 2 : ti); ++tj)
          tiles.push_back(TileDesc{vc, uint16_t(ti), uint16_t(tj)});
    }
  }
  auto p = std::make_unique<Plan>();
  p->num_tiles = int(tiles.size());
  p->num_chans = batch;
  cudaError_t e = cudaMalloc(&p->d_tiles, tiles.size() * sizeof(TileDesc));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_chans, chans.size() * sizeof(ChanDesc));
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_tiles, tiles.data(), tiles.size() * sizeof(TileDesc),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_chans, chans.data(), chans.size() * sizeof(ChanDesc),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(h, e, "tile plan upload");
  *out = p.get();
  h->plans.emplace(key, std::move(p));
  return FTDX_OK;
}

int pair_grid_limit(ftdx_handle h) {
  if (h->pair_grid < 0) {
    int clusters = 0;
    if (herk_fp8_pair_max_clusters(h->sm_count, &clusters) != cudaSuccess) {
      cudaGetLastError();
      clusters = 0;
    }
    h->pair_grid = 2 * std::min(clusters, h->sm_count / 2);
    if (h->verbosity > 0) fprintf(stderr, "ftdx: %d co-resident CTA pairs\n", h->pair_grid / 2);
  }
  return h->pair_grid;
}

// Tensor map over the operand planes Z[nplanes][rows][Kp] (bytes): box of
// 128 samples x box_rows rows x 1 plane, 128-byte swizzle.
ftdx_status encode_planes_map(ftdx_handle h, uint8_t* z, int64_t rows, int64_t Kp,
                              CUtensorMap* tm, int box_rows, int nplanes, bool fp6) {
  auto enc = get_encode_fn();
  if (!enc) return fail(h, FTDX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const cuuint32_t estr[3] = {1, 1, 1};
  // fp6: Kp packed 6-bit codes per row (3 Kp / 4 bytes; Kp is a multiple of
  // 128, so the row pitch is a multiple of 32 bytes as the 16 x U6 type needs),
  // unpacked by the TMA to one byte per code in shared memory
  const int64_t pitch = fp6 ? Kp / 4 * 3 : Kp;
  const cuuint64_t dims[3] = {cuuint64_t(Kp), cuuint64_t(rows), cuuint64_t(nplanes)};
  const cuuint64_t strides[2] = {cuuint64_t(pitch), cuuint64_t(rows * pitch)};
  const cuuint32_t box[3] = {cuuint32_t(kStageK), cuuint32_t(box_rows), 1};
  CUresult r = enc(tm, fp6 ? CU_TENSOR_MAP_DATA_TYPE_16U6_ALIGN16B : CU_TENSOR_MAP_DATA_TYPE_UINT8,
                   3, z, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, FTDX_ERR_CUDA, "tensor map encode failed: %d", int(r));
  return FTDX_OK;
}

ftdx_status encode_qc_map(ftdx_handle h, const void* qc, int64_t rows, int K, CUtensorMap* tm) {
  auto enc = get_encode_fn();
  if (!enc) return fail(h, FTDX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const cuuint32_t estr[2] = {1, 1};
  const cuuint64_t dims[2] = {cuuint64_t(K), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(K)};
  const cuuint32_t box[2] = {cuuint32_t(kStageK), cuuint32_t(kTile)};
  CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(qc), dims, strides, box,
                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, FTDX_ERR_CUDA, "QC tensor map encode failed: %d", int(r));
  return FTDX_OK;
}

static cudaEvent_t pool_event(ftdx_handle h) {
  if (!h->event_pool.empty()) {
    cudaEvent_t e = h->event_pool.back();
    h->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

ScopedTimer::ScopedTimer(ftdx_handle h_, cudaStream_t s_, int kind_) : h(h_), s(s_), kind(kind_) {
  if (h->profiling && !stream_capturing(s)) {
    a = pool_event(h);
    cudaEventRecord(a, s);
  }
}

ScopedTimer::~ScopedTimer() {
  if (a) {
    cudaEvent_t b = pool_event(h);
    cudaEventRecord(b, s);
    h->timed.push_back({a, b, kind});
  }
}

}  // namespace ftdx

using namespace ftdx;

extern "C" {

int ftdx_version(void) { return (FTDX_VERSION_MAJOR << 16) | FTDX_VERSION_MINOR; }

const char* ftdx_status_string(ftdx_status s) {
  switch (s) {
    case FTDX_OK: return "success";
    case FTDX_ERR_INVALID_ARG: return "invalid argument";
    case FTDX_ERR_UNSUPPORTED: return "unsupported request";
    case FTDX_ERR_CUDA: return "CUDA error";
    case FTDX_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case FTDX_ERR_ALLOC: return "workspace allocation failed";
    case FTDX_ERR_CAPACITY: return "workspace too small during graph capture";
    case FTDX_ERR_TIMEOUT: return "device-side wait timed out";
    case FTDX_ERR_CACHE: return "tune cache error";
  }
  return "unknown status";
}

ftdx_status ftdx_create(ftdx_handle* out, const ftdx_config* cfg) {
  if (!out) return FTDX_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return FTDX_ERR_NO_DEVICE;
  }
  int dev = (cfg && cfg->device >= 0) ? cfg->device : -1;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return FTDX_ERR_NO_DEVICE;
  if (dev >= ndev) return FTDX_ERR_INVALID_ARG;
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return FTDX_ERR_NO_DEVICE;
  if (prop.major != 10 || prop.minor != 0) return FTDX_ERR_NO_DEVICE;
  if (cudaSetDevice(dev) != cudaSuccess) return FTDX_ERR_NO_DEVICE;
  auto* h = new ftdx_context();
  h->device = dev;
  h->sm_count = prop.multiProcessorCount;
  h->device_name = prop.name;
  for (char& c : h->device_name)
    if (c == ' ' || c == '\t') c = '_';
  if (cfg) h->verbosity = cfg->verbosity;
  if (cfg && cfg->tune_cache)
    h->tune_cache = cfg->tune_cache;
  else if (const char* env = getenv("FTDX_TUNE_CACHE"))
    h->tune_cache = env;
  if (cudaMalloc(&h->d_status, sizeof(uint32_t)) != cudaSuccess ||
      cudaMemset(h->d_status, 0, sizeof(uint32_t)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    if (h->d_status) cudaFree(h->d_status);
    delete h;
    return FTDX_ERR_ALLOC;
  }
  load_tune_cache(h);
  *out = h;
  return FTDX_OK;
}

ftdx_status ftdx_destroy(ftdx_handle h) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  cudaDeviceSynchronize();
  release_graphs(h);
  h->plans.clear();
  h->vplans.clear();
  for (auto& t : h->timed) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  for (auto e : h->event_pool) cudaEventDestroy(e);
  if (h->z) cudaFree(h->z);
  if (h->aux) cudaFree(h->aux);
  if (h->split_ws) cudaFree(h->split_ws);
  if (h->strided_ws) cudaFree(h->strided_ws);
  if (h->d_status) cudaFree(h->d_status);
  if (h->capture_stream) cudaStreamDestroy(h->capture_stream);
  delete h;
  return FTDX_OK;
}

const char* ftdx_last_error(ftdx_handle h) {
  if (h) return h->last_error.c_str();
  const std::string& t = ftdx::thread_error();
  return t.empty() ? "null handle" : t.c_str();
}

ftdx_status ftdx_device_status(ftdx_handle h, void* stream, uint32_t* bits) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamSynchronize");
  uint32_t v = 0;
  e = cudaMemcpy(&v, h->d_status, sizeof(v), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(h, e, "status read");
  cudaMemset(h->d_status, 0, sizeof(uint32_t));
  if (bits) *bits = v;
  if (v) return fail(h, FTDX_ERR_TIMEOUT, "device status 0x%x", v);
  return FTDX_OK;
}

ftdx_status ftdx_set_profiling(ftdx_handle h, int enable) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  h->profiling = enable != 0;
  return FTDX_OK;
}

ftdx_status ftdx_profile_read(ftdx_handle h, double* herk_ms, int* herk_launches, double* prep_ms,
                              int* prep_launches) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  double ms[2] = {0, 0};
  int n[2] = {0, 0};
  ftdx_status st = FTDX_OK;
  for (auto& t : h->timed) {
    float v = 0.f;
    cudaError_t e = cudaEventSynchronize(t.b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&v, t.a, t.b);
    if (e != cudaSuccess) st = cuda_fail(h, e, "profile event");
    ms[t.kind] += v;
    n[t.kind] += 1;
    h->event_pool.push_back(t.a);
    h->event_pool.push_back(t.b);
  }
  h->timed.clear();
  if (herk_ms) *herk_ms = ms[0];
  if (herk_launches) *herk_launches = n[0];
  if (prep_ms) *prep_ms = ms[1];
  if (prep_launches) *prep_launches = n[1];
  return st;
}

}  // extern "C"
