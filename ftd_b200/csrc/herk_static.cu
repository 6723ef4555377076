// herk_static.cu -- a correlator entry point that never allocates memory.
//
// Some callers cannot let a library allocate GPU memory once they are
// running: a real-time X-engine that sizes every buffer when an observation
// starts and must not stall (or fail) mid-stream on a cudaMalloc; a host
// framework whose device memory all comes from its own pool, where a stray
// cudaMalloc breaks its accounting or is forbidden outright; an embedded
// deployment with a fixed memory budget.  ftdx_herk_static serves them: it
// runs the same promotion and tcgen05 correlator kernels as ftdx_herk, but
// keeps all of their scratch (the FP8 operand planes, the tile list, the
// channel table and the device status word) in one file-scope __device__
// array of FTDX_STATIC_SCRATCH_BYTES, which every GPU that loads this
// library holds until the process exits.  The caller passes only the input
// voltages and the output triangles.
#include <algorithm>
#include <cmath>
#include <mutex>

#include <cudaTypedefs.h>

#include "../../include/ftdx.h"
#include "herk_fp8.cuh"

namespace ftdx {
namespace {

constexpr size_t kStaticBytes = size_t(FTDX_STATIC_SCRATCH_BYTES);
constexpr size_t kStatusOffset = 0;      // uint32_t device status word
constexpr size_t kPlanOffset = 256;      // ChanDesc[batch] then TileDesc[tiles]
constexpr int kMaxDevices = 64;

// The scratch itself.  In host code this name is only a stand-in symbol, not
// a device address: the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint8_t g_static_scratch[kStaticBytes];

std::mutex g_setup_mutex;
uint8_t* g_scratch_ptr[kMaxDevices] = {};

// Fills the channel table and the lower-triangle tile list (ti-major, tj <= ti,
// channel-major: the order ftdx_herk uses) and clears the status word.
__global__ void static_plan_kernel(ChanDesc* chans, TileDesc* tiles, uint32_t* status, int n,
                                   int kblocks, int batch, int per_chan) {
  const int64_t total = int64_t(batch) * per_chan;
  const int64_t P = int64_t(n) * (n + 1) / 2;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += int64_t(gridDim.x) * blockDim.x) {
    const int c = int(t / per_chan);
    const int r = int(t - int64_t(c) * per_chan);
    int ti = int((sqrtf(8.f * float(r) + 1.f) - 1.f) * 0.5f);
    while (ti > 0 && ti * (ti + 1) / 2 > r) --ti;
    while ((ti + 1) * (ti + 2) / 2 <= r) ++ti;
    const int tj = r - ti * (ti + 1) / 2;
    tiles[t] = TileDesc{c, uint16_t(ti), uint16_t(tj)};
    if (r == 0) chans[c] = ChanDesc{n, kblocks, int64_t(c) * n, int64_t(c) * P, 0};
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *status = 0u;
}

// One-time set-up per device, with that device current: the device address
// of the scratch array.
cudaError_t scratch_for_device(int dev, uint8_t** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<uint8_t*>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

}  // namespace
}  // namespace ftdx

using namespace ftdx;

extern "C" ftdx_status ftdx_herk_static(const void* A, void* C, int N, int K, int batch,
                                        void* stream, uint32_t* status_out, size_t* scratch_used) {
  if (!A || !C || N < 1 || K < 1 || batch < 1) {
    set_thread_error("ftdx_herk_static: null pointer or size < 1");
    return FTDX_ERR_INVALID_ARG;
  }
  if ((reinterpret_cast<uintptr_t>(C) & 7) != 0) {
    set_thread_error("ftdx_herk_static: C is not 8-byte aligned");
    return FTDX_ERR_INVALID_ARG;
  }
  if (N > 65535 * kTile || int64_t(K) > (int64_t(1) << 30)) {
    set_thread_error("ftdx_herk_static: N=%d or K=%d out of range", N, K);
    return FTDX_ERR_INVALID_ARG;
  }
  // Scratch layout: status | channel table + tile list | FP8 planes (1 KiB
  // aligned).  All sizes in 64 bits: the tile count of a large N overflows int.
  const int64_t Kp = (int64_t(K) + kStageK - 1) / kStageK * kStageK;
  const int64_t rows = int64_t(N) * batch;
  const int64_t nb = (int64_t(N) + kTile - 1) / kTile;
  const int64_t per_chan = nb * (nb + 1) / 2;
  const int64_t ntiles = int64_t(batch) * per_chan;
  const uint64_t plan_bytes =
      uint64_t(batch) * sizeof(ChanDesc) + uint64_t(ntiles) * sizeof(TileDesc);
  const uint64_t z_off = (kPlanOffset + plan_bytes + 1023) / 1024 * 1024;
  const uint64_t need = z_off + uint64_t(2) * uint64_t(rows) * uint64_t(Kp);
  if (scratch_used) *scratch_used = size_t(need);
  if (need > kStaticBytes) {
    set_thread_error(
        "ftdx_herk_static: N=%d K=%d batch=%d needs %llu bytes of scratch; the static scratch "
        "holds %zu (FTDX_STATIC_SCRATCH_BYTES)",
        N, K, batch, static_cast<unsigned long long>(need), kStaticBytes);
    return FTDX_ERR_CAPACITY;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (status_out) {
    // reading the status synchronises the stream, which a capture forbids
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      set_thread_error("ftdx_herk_static: status_out must be NULL while the stream is captured");
      return FTDX_ERR_INVALID_ARG;
    }
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    set_thread_error("ftdx_herk_static: no current CUDA device");
    return FTDX_ERR_NO_DEVICE;
  }
  int major = 0, sms = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (major != 10) {
    set_thread_error("ftdx_herk_static: device %d is not an sm_100 GPU", dev);
    return FTDX_ERR_NO_DEVICE;
  }
  uint8_t* base = nullptr;
  const cudaError_t se = scratch_for_device(dev, &base);
  if (se != cudaSuccess) {
    set_thread_error("ftdx_herk_static: cudaGetSymbolAddress: %s", cudaGetErrorString(se));
    return FTDX_ERR_CUDA;
  }

  uint32_t* status = reinterpret_cast<uint32_t*>(base + kStatusOffset);
  ChanDesc* chans = reinterpret_cast<ChanDesc*>(base + kPlanOffset);
  TileDesc* tiles = reinterpret_cast<TileDesc*>(base + kPlanOffset + size_t(batch) * sizeof(ChanDesc));
  uint8_t* z = base + z_off;

  const int pblocks = int(std::min<int64_t>((ntiles + 255) / 256, int64_t(sms) * 4));
  static_plan_kernel<<<pblocks, 256, 0, s>>>(chans, tiles, status, N, int(Kp / kStageK), batch,
                                             int(per_chan));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = launch_qc_to_planes(static_cast<const uint8_t*>(A), z, rows, K, int(Kp), s);
  if (e != cudaSuccess) {
    set_thread_error("ftdx_herk_static: launch failed: %s", cudaGetErrorString(e));
    return FTDX_ERR_CUDA;
  }

  auto enc = encode_fn();
  if (!enc) {
    set_thread_error("ftdx_herk_static: cuTensorMapEncodeTiled unavailable");
    return FTDX_ERR_CUDA;
  }
  CUtensorMap tm;
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint64_t dims[3] = {cuuint64_t(Kp), cuuint64_t(rows), 2};
  const cuuint64_t strides[2] = {cuuint64_t(Kp), cuuint64_t(rows * Kp)};
  const cuuint32_t box[3] = {cuuint32_t(kStageK), cuuint32_t(kTile), 1};
  if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, z, dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
    set_thread_error("ftdx_herk_static: tensor map encode failed");
    return FTDX_ERR_CUDA;
  }

  HerkArgs args = herk_args_default();
  args.tiles = tiles;
  args.chans = chans;
  args.num_tiles = int(ntiles);
  args.out_fp16 = 0;
  args.bulk_store = 0;
  args.out_format = 0;
  args.out = C;
  args.alpha = 1.f;
  args.beta = 0.f;
  args.status = status;
  const int grid = int(std::min<int64_t>(ntiles, sms));
  e = launch_herk_fp8(tm, args, grid, s);
  if (e != cudaSuccess) {
    set_thread_error("ftdx_herk_static: correlator launch failed: %s", cudaGetErrorString(e));
    return FTDX_ERR_CUDA;
  }

  if (status_out) {
    // an ordered copy on the caller's stream, so no other stream is waited on
    uint32_t v = 0;
    e = cudaMemcpyAsync(&v, status, sizeof(v), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      set_thread_error("ftdx_herk_static: status read failed: %s", cudaGetErrorString(e));
      return FTDX_ERR_CUDA;
    }
    *status_out = v;
    if (v) {
      set_thread_error("ftdx_herk_static: device status bits 0x%x (a bounded wait ran out)", v);
      return FTDX_ERR_TIMEOUT;
    }
  }
  return FTDX_OK;
}
