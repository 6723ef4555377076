// peak_probe.cu -- dense tensor-core throughput of this GPU, measured with the
// MMA shapes the correlators issue, for the roofline denominators: a cluster of
// two CTAs per SM pair issues back-to-back tcgen05.mma.cta_group::2 of
// M = 256, N = 256 (FP8 E4M3, K = 32; or NVFP4 block16, K = 64) from fixed
// zero-filled shared-memory tiles into one TMEM accumulator, with no loads
// and no epilogue.  Achieved rate = 2 M N K x MMAs x pairs / time.
#include "herk_fp8.cuh"
#include "sm100.cuh"
#include "../../include/ftdx.h"
#include "context.h"

namespace ftdx {
namespace {

constexpr int kProbeTile = 128 * 128;              // bytes: 128 rows x 128 B (SW128)
// more shared memory than two CTAs can share, so one CTA (and one 512-column
// TMEM allocation) per SM; the tiles use the first 37 KB
constexpr size_t kProbeSmem = 120 * 1024;
static_assert(1024 + 2 * kProbeTile + 4096 + 256 <= kProbeSmem, "probe layout");

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(128, 1)
    peak_probe_kernel(int kind, int iters, uint32_t* status) {
  extern __shared__ uint8_t smem_dyn[];
  uint8_t* smem = smem_dyn + ((1024u - (dev::smem_u32(smem_dyn) & 1023u)) & 1023u);
  uint8_t* sf = smem + 2 * kProbeTile;  // 4 KB of zero scale factors
  uint64_t* bar = reinterpret_cast<uint64_t*>(sf + 4096);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool leader = dev::cluster_rank() == 0;
  for (int x = threadIdx.x; x < (2 * kProbeTile + 4096) / 16; x += blockDim.x)
    reinterpret_cast<uint4*>(smem)[x] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    dev::mbar_init(dev::smem_u32(bar), 1);
    dev::fence_mbar_init();
  }
  dev::fence_proxy_async_smem();
  if (warp == 0) {
    dev::tmem_alloc_pair(dev::smem_u32(tmem_slot), 512);
    dev::tmem_relinquish_pair();
  }
  dev::tc_fence_before();
  __syncthreads();
  dev::cluster_sync_all();
  dev::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  if (warp == 0 && lane == 0 && leader) {
    const uint64_t a = dev::sdesc_sw128_kmajor(dev::smem_u32(smem));
    const uint64_t b = dev::sdesc_sw128_kmajor(dev::smem_u32(smem) + kProbeTile);
    if (kind == 0) {
      const uint32_t idesc = dev::idesc_f32acc(dev::kFmtE4M3, dev::kFmtE4M3, 256, 256);
      for (int it = 0; it < iters; ++it) dev::mma_f8f6f4_pair(tmem, a, b, idesc, it > 0);
    } else {
      // scale factors: SFA 4 columns, SFB 8 columns (256 B rows) after the accumulator
      const uint32_t sfa = tmem + 256, sfb = tmem + 264;
      dev::tmem_cp_32x128b_warpx4_pair(sfa, dev::sdesc_none_kmajor(dev::smem_u32(sf), 128));
      dev::tmem_cp_32x128b_warpx4_pair(sfb, dev::sdesc_none_kmajor(dev::smem_u32(sf) + 512, 128));
      dev::tmem_cp_32x128b_warpx4_pair(sfb + 4,
                                       dev::sdesc_none_kmajor(dev::smem_u32(sf) + 1024, 128));
      const uint32_t idesc = (1u << 7) | (1u << 10) | ((256u >> 3) << 17) | ((256u >> 4) << 24);
      for (int it = 0; it < iters; ++it) dev::mma_nvf4_pair(tmem, a, b, idesc, sfa, sfb, it > 0);
    }
    dev::mma_commit_pair(dev::smem_u32(bar));
    dev::mma_commit_pair(dev::map_shared(dev::smem_u32(bar), 1));
  }
  // every thread of both CTAs waits for the MMAs (bounded)
  volatile int never = 0;
  if (!dev::mbar_wait(dev::smem_u32(bar), 0, &never)) {
    if (threadIdx.x == 0) atomicOr(status, dev::kStatusTimeoutOther);
  }
  dev::tc_fence_before();
  __syncthreads();
  dev::cluster_sync_all();
  if (warp == 0) {
    dev::tc_fence_after();
    dev::tmem_dealloc_pair(tmem, 512);
  }
}

}  // namespace
}  // namespace ftdx

using namespace ftdx;

extern "C" ftdx_status ftdx_peak_probe(ftdx_handle h, int kind, int iters, int reps, double* tflops) {
  if (!h || !tflops || (kind != 0 && kind != 1) || iters < 1 || reps < 1)
    return FTDX_ERR_INVALID_ARG;
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  e = ensure_smem_limit(reinterpret_cast<const void*>(peak_probe_kernel), kProbeSmem);
  if (e != cudaSuccess) return cuda_fail(h, e, "probe attributes");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(h->sm_count & ~1), 1, 1);
  cfg.blockDim = dim3(128, 1, 1);
  cfg.dynamicSmemBytes = kProbeSmem;
  int clusters = 0;
  e = cudaOccupancyMaxActiveClusters(&clusters, peak_probe_kernel, &cfg);
  if (e != cudaSuccess || clusters < 1) return cuda_fail(h, e, "probe occupancy");
  if (clusters > h->sm_count / 2) clusters = h->sm_count / 2;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaStream_t s = nullptr;
  float best = 1e30f;
  for (int r = 0; r < reps + 1; ++r) {  // the first launch warms up
    cudaEventRecord(a, s);
    peak_probe_kernel<<<2 * clusters, 128, kProbeSmem, s>>>(kind, iters, h->d_status);
    cudaEventRecord(b, s);
    e = cudaEventSynchronize(b);
    if (e != cudaSuccess) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (r > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) return cuda_fail(h, e, "probe launch");
  const double k = kind == 0 ? 32.0 : 64.0;
  const double flop = 2.0 * 256.0 * 256.0 * k * double(iters) * double(clusters);
  *tflops = flop / (double(best) * 1e-3) / 1e12;
  return FTDX_OK;
}
