// ftdx_api.cu -- C ABI of the correlator: handles, workspace, tile plans,
// tensor-map encoding and kernel dispatch.  See include/ftdx.h.
#include "../../include/ftdx.h"
#include "herk_fp8.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

namespace {

using ftdx::ChanDesc;
using ftdx::TileDesc;

PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Device-resident tile list + channel table for one problem shape.
struct Plan {
  TileDesc* d_tiles = nullptr;
  ChanDesc* d_chans = nullptr;
  int num_tiles = 0;
  int num_chans = 0;
  ~Plan() {
    if (d_tiles) cudaFree(d_tiles);
    if (d_chans) cudaFree(d_chans);
  }
};

}  // namespace

struct ftdx_context {
  int device = 0;
  int sm_count = 148;
  int verbosity = 0;
  std::string tune_cache;
  std::string last_error;
  uint8_t* z = nullptr;       // FP8 operand workspace
  size_t z_cap = 0;
  bool z_reserved = false;    // sized by ftdx_init_herk
  uint32_t* d_status = nullptr;
  std::map<std::tuple<int, int, int>, std::unique_ptr<Plan>> plans;  // (N, kblocks, batch)
  int bulk_store = 0;  // epilogue store mode (HerkArgs::bulk_store)
  // kernel timing (ftdx_set_profiling)
  bool profiling = false;
  struct Timed {
    cudaEvent_t a, b;
    int kind;  // 0 = herk, 1 = prep
  };
  std::vector<Timed> timed;
  std::vector<cudaEvent_t> event_pool;
};

namespace {

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
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess) return false;
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
    cudaStreamSynchronize(s);
    cudaFree(h->z);
    h->z = nullptr;
    h->z_cap = 0;
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

// Lower-triangle tile list for `batch` channels of N inputs, channel-major so
// that consecutive CTAs share a channel's operand in L2.
ftdx_status get_plan(ftdx_handle h, int N, int kblocks, int batch, cudaStream_t s,
                     const Plan** out) {
  auto key = std::make_tuple(N, kblocks, batch);
  auto it = h->plans.find(key);
  if (it != h->plans.end()) {
    *out = it->second.get();
    return FTDX_OK;
  }
  if (stream_capturing(s))
    return fail(h, FTDX_ERR_CAPACITY,
                "tile plan for N=%d batch=%d built while capturing; call ftdx_init_herk first", N,
                batch);
  const int nb = (N + ftdx::kTile - 1) / ftdx::kTile;
  std::vector<ChanDesc> chans(batch);
  std::vector<TileDesc> tiles;
  tiles.reserve(size_t(batch) * nb * (nb + 1) / 2);
  for (int c = 0; c < batch; ++c) {
    chans[c].n = N;
    chans[c].kblocks = kblocks;
    chans[c].row0 = int64_t(c) * N;
    chans[c].out0 = int64_t(c) * (int64_t(N) * (N + 1) / 2);
    chans[c].reserved = 0;
    for (int ti = 0; ti < nb; ++ti)
      for (int tj = 0; tj <= ti; ++tj) tiles.push_back(TileDesc{c, uint16_t(ti), uint16_t(tj)});
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

// Tensor map over the operand planes Z[2][rows][Kp] (bytes): box of
// 128 samples x 128 rows x 1 plane, 128-byte swizzle.
ftdx_status encode_planes_map(ftdx_handle h, uint8_t* z, int64_t rows, int64_t Kp,
                              CUtensorMap* tm) {
  auto enc = get_encode_fn();
  if (!enc) return fail(h, FTDX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint64_t dims[3] = {cuuint64_t(Kp), cuuint64_t(rows), 2};
  const cuuint64_t strides[2] = {cuuint64_t(Kp), cuuint64_t(rows * Kp)};
  const cuuint32_t box[3] = {cuuint32_t(ftdx::kStageK), cuuint32_t(ftdx::kTile), 1};
  CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, z, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, FTDX_ERR_CUDA, "tensor map encode failed: %d", int(r));
  return FTDX_OK;
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

cudaEvent_t pool_event(ftdx_handle h) {
  if (!h->event_pool.empty()) {
    cudaEvent_t e = h->event_pool.back();
    h->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records an event pair around one kernel launch when profiling is on.
struct ScopedTimer {
  ftdx_handle h;
  cudaStream_t s;
  int kind;
  cudaEvent_t a = nullptr;
  ScopedTimer(ftdx_handle h_, cudaStream_t s_, int kind_) : h(h_), s(s_), kind(kind_) {
    if (h->profiling) {
      a = pool_event(h);
      cudaEventRecord(a, s);
    }
  }
  ~ScopedTimer() {
    if (a) {
      cudaEvent_t b = pool_event(h);
      cudaEventRecord(b, s);
      h->timed.push_back({a, b, kind});
    }
  }
};

}  // namespace

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
  int major = 0, minor = 0, sms = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (major != 10 || minor != 0) return FTDX_ERR_NO_DEVICE;
  if (cudaSetDevice(dev) != cudaSuccess) return FTDX_ERR_NO_DEVICE;
  auto* h = new ftdx_context();
  h->device = dev;
  h->sm_count = sms;
  if (cfg) {
    h->verbosity = cfg->verbosity;
    if (cfg->tune_cache) h->tune_cache = cfg->tune_cache;
  }
  if (cudaMalloc(&h->d_status, sizeof(uint32_t)) != cudaSuccess ||
      cudaMemset(h->d_status, 0, sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return FTDX_ERR_ALLOC;
  }
  *out = h;
  return FTDX_OK;
}

ftdx_status ftdx_destroy(ftdx_handle h) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  cudaDeviceSynchronize();
  h->plans.clear();
  for (auto& t : h->timed) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  for (auto e : h->event_pool) cudaEventDestroy(e);
  if (h->z) cudaFree(h->z);
  if (h->d_status) cudaFree(h->d_status);
  delete h;
  return FTDX_OK;
}

const char* ftdx_last_error(ftdx_handle h) { return h ? h->last_error.c_str() : "null handle"; }

ftdx_status ftdx_init_herk(ftdx_handle h, int N, int K, int batch, void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (N < 1 || K < 1 || batch < 1) return fail(h, FTDX_ERR_INVALID_ARG, "init_herk: bad sizes");
  cudaSetDevice(h->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t Kp = round_up(K, ftdx::kStageK);
  ftdx_status st = ensure_workspace(h, size_t(2) * N * batch * Kp, s);
  if (st != FTDX_OK) return st;
  h->z_reserved = true;
  const Plan* p = nullptr;
  return get_plan(h, N, int(Kp / ftdx::kStageK), batch, s, &p);
}

ftdx_status ftdx_end_herk(ftdx_handle h) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  cudaSetDevice(h->device);
  cudaDeviceSynchronize();
  if (h->z) cudaFree(h->z);
  h->z = nullptr;
  h->z_cap = 0;
  h->z_reserved = false;
  h->plans.clear();
  return FTDX_OK;
}

ftdx_status ftdx_herk(ftdx_handle h, const void* A, void* C, int N, int K, int batch,
                      ftdx_input input, ftdx_compute compute, ftdx_output output,
                      ftdx_format format, float alpha, float beta, void* stream, int tune) {
  (void)tune;
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!A || !C) return fail(h, FTDX_ERR_INVALID_ARG, "herk: null A or C");
  if (N < 1 || K < 1 || batch < 1)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: N, K and batch must be >= 1 (got %d, %d, %d)", N,
                K, batch);
  if (input != FTDX_IN_INT4 && input != FTDX_IN_FP16)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: bad input precision %d", int(input));
  if (output != FTDX_OUT_FP32 && output != FTDX_OUT_FP16)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: bad output precision %d", int(output));
  if (format != FTDX_FORMAT_PACKED_TRIANGLE)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: only the packed triangle format exists");
  if (compute != FTDX_COMPUTE_FP8)
    return fail(h, FTDX_ERR_UNSUPPORTED, "herk: compute precision %d not implemented",
                int(compute));
  if ((reinterpret_cast<uintptr_t>(C) & (output == FTDX_OUT_FP32 ? 7 : 3)) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: C is not aligned to one complex element");
  if (input == FTDX_IN_FP16 && (reinterpret_cast<uintptr_t>(A) & 3) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: FP16 A must be 4-byte aligned");
  // Row coordinates of the TMA boxes are 32-bit.
  if (int64_t(N) * batch + 256 > (int64_t(1) << 31))
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: N*batch too large for one call");
  if (N > 65535 * ftdx::kTile)
    return fail(h, FTDX_ERR_INVALID_ARG, "herk: N too large");

  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t Kp = round_up(K, ftdx::kStageK);
  const int64_t rows = int64_t(N) * batch;
  ftdx_status st = ensure_workspace(h, size_t(2 * rows * Kp), s);
  if (st != FTDX_OK) return st;
  const Plan* plan = nullptr;
  st = get_plan(h, N, int(Kp / ftdx::kStageK), batch, s, &plan);
  if (st != FTDX_OK) return st;

  {
    ScopedTimer tm(h, s, 1);
    if (input == FTDX_IN_INT4)
      e = ftdx::launch_qc_to_planes(static_cast<const uint8_t*>(A), h->z, rows, K, int(Kp), s);
    else
      e = ftdx::launch_fp16_to_planes(A, h->z, rows, K, int(Kp), s);
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "operand promotion launch");

  CUtensorMap tmZ;
  st = encode_planes_map(h, h->z, rows, Kp, &tmZ);
  if (st != FTDX_OK) return st;
  ftdx::HerkArgs args;
  args.tiles = plan->d_tiles;
  args.chans = plan->d_chans;
  args.num_tiles = plan->num_tiles;
  args.out_fp16 = (output == FTDX_OUT_FP16) ? 1 : 0;
  args.bulk_store = h->bulk_store;
  args.reserved = 0;
  args.out = C;
  args.alpha = alpha;
  args.beta = beta;
  args.status = h->d_status;
  const int grid = plan->num_tiles < h->sm_count ? plan->num_tiles : h->sm_count;
  {
    ScopedTimer tm(h, s, 0);
    e = ftdx::launch_herk_fp8(tmZ, args, grid, s);
  }
  if (e != cudaSuccess) return cuda_fail(h, e, "HERK kernel launch");
  return FTDX_OK;
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
