// peak_probe.cu -- dense tensor-core throughput of this GPU, measured with the
// MMA shapes the correlators issue, for the roofline denominators.  No loads
// and no epilogue; achieved rate = 2 M N K x MMAs x issuers / time.
//  * kind 0 / 1: a cluster of two CTAs per SM pair issues back-to-back
//    tcgen05.mma.cta_group::2 of M = 256, N = 256 (FP8 E4M3, K = 32; or NVFP4
//    block16, K = 64) from fixed zero-filled shared-memory tiles into one
//    TMEM accumulator.
//  * kind 2: the CTA-pair correlator's MMA stream (two M = N = 256 FP8 MMAs
//    per 32 samples, A = Re_j / Im_j, B = the two 128-row halves) on
//    QC-valued operands: E4M3 codes of random integers -7..7, as the
//    promotion writes them, cycling the four 32-byte K slices of the tiles.
//  * kind 3: the single-CTA correlator's MMA stream (four M = N = 128 FP8 MMAs
//    per 32 samples into a Re and an Im accumulator, the fourth negated) on
//    the same QC-valued operands, one CTA per SM, cta_group::1.
// Zero tiles draw less power than data does, so kinds 2 and 3 are the
// ceilings with the correlator's own operand values.
#include "herk_fp8.cuh"
#include "qc_codec.cuh"
#include "sm100.cuh"
#include "../../include/ftdx.h"
#include "context.h"

namespace ftdx {
namespace {

constexpr int kProbeTile = 128 * 128;              // bytes: 128 rows x 128 B (SW128)
constexpr int kProbeTiles = 4;                     // kinds 2, 3: A_re, A_im, B halves
// more shared memory than two CTAs can share, so one CTA (and one 512-column
// TMEM allocation) per SM; tiles, then 4 KB of scale factors, then the barrier
constexpr size_t kProbeSmem = 120 * 1024;
static_assert(1024 + kProbeTiles * kProbeTile + 4096 + 256 <= kProbeSmem, "probe layout");

// Fill the tiles with zeros (kinds 0, 1) or with E4M3 codes of QC-valued
// samples (integers -7..7) from a per-CTA integer hash.
__device__ void probe_fill(uint8_t* smem, int kind) {
  const uint32_t seed = 0x9E3779B9u * (blockIdx.x + 1u);
  for (int x = threadIdx.x; x < (kProbeTiles * kProbeTile + 4096) / 4; x += blockDim.x) {
    uint32_t v = 0;
    if (kind >= 2 && x < kProbeTiles * kProbeTile / 4) {
      uint32_t hsh = seed ^ (uint32_t(x) * 0x85EBCA6Bu);
      hsh ^= hsh >> 13;
      hsh *= 0xC2B2AE35u;
      hsh ^= hsh >> 16;
      uint32_t im;
      qc4_to_e4m3(hsh, v, im);
      v ^= im & 0x80808080u;  // a sign pattern independent of the magnitudes
    }
    reinterpret_cast<uint32_t*>(smem)[x] = v;
  }
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(128, 1)
    peak_probe_kernel(int kind, int iters, uint32_t* status) {
  extern __shared__ uint8_t smem_dyn[];
  uint8_t* smem = smem_dyn + ((1024u - (dev::smem_u32(smem_dyn) & 1023u)) & 1023u);
  uint8_t* sf = smem + kProbeTiles * kProbeTile;  // 4 KB of zero scale factors
  uint64_t* bar = reinterpret_cast<uint64_t*>(sf + 4096);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool leader = dev::cluster_rank() == 0;
  probe_fill(smem, kind);
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
    } else if (kind == 2) {
      // the pair kernel's k-step: (A = Re_j, B = X), (A = Im_j, B = Y); iters MMAs
      const uint32_t idesc = dev::idesc_f32acc(dev::kFmtE4M3, dev::kFmtE4M3, 256, 256);
      const uint32_t t0 = dev::smem_u32(smem);
      for (int it = 0; it < iters; it += 2) {
        const uint32_t ks = 32u * uint32_t((it >> 1) & 3);
        dev::mma_f8f6f4_pair(tmem, dev::sdesc_sw128_kmajor(t0 + ks),
                             dev::sdesc_sw128_kmajor(t0 + 2 * kProbeTile + ks), idesc, it > 0);
        dev::mma_f8f6f4_pair(tmem, dev::sdesc_sw128_kmajor(t0 + kProbeTile + ks),
                             dev::sdesc_sw128_kmajor(t0 + 3 * kProbeTile + ks), idesc, 1);
      }
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
    dev::mma_commit_pair_both(dev::smem_u32(bar));
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

// Kind 3: one CTA per SM, cta_group::1 throughout.  The single-CTA
// correlator's k-step: Re += A_re B_re, Im += A_re B_im, Re += A_im B_im,
// Im -= A_im B_re (M = N = 128, K = 32); iters MMAs per CTA.
__global__ void __launch_bounds__(128, 1) peak_probe_single_kernel(int iters, uint32_t* status) {
  extern __shared__ uint8_t smem_dyn[];
  uint8_t* smem = smem_dyn + ((1024u - (dev::smem_u32(smem_dyn) & 1023u)) & 1023u);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kProbeTiles * kProbeTile + 4096);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  probe_fill(smem, 3);
  if (threadIdx.x == 0) {
    dev::mbar_init(dev::smem_u32(bar), 1);
    dev::fence_mbar_init();
  }
  dev::fence_proxy_async_smem();
  if (warp == 0) {
    dev::tmem_alloc(dev::smem_u32(tmem_slot), 512);
    dev::tmem_relinquish();
  }
  dev::tc_fence_before();
  __syncthreads();
  dev::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  if (warp == 0 && lane == 0) {
    const uint32_t idesc = dev::idesc_f32acc(dev::kFmtE4M3, dev::kFmtE4M3, 128, 128);
    const uint32_t idesc_neg = dev::idesc_f32acc(dev::kFmtE4M3, dev::kFmtE4M3, 128, 128, 1);
    const uint32_t t0 = dev::smem_u32(smem);
    const uint32_t d_re = tmem, d_im = tmem + 128;
    for (int it = 0; it < iters; it += 4) {
      const uint32_t ks = 32u * uint32_t((it >> 2) & 3);
      const uint64_t are = dev::sdesc_sw128_kmajor(t0 + ks);
      const uint64_t aim = dev::sdesc_sw128_kmajor(t0 + kProbeTile + ks);
      const uint64_t bre = dev::sdesc_sw128_kmajor(t0 + 2 * kProbeTile + ks);
      const uint64_t bim = dev::sdesc_sw128_kmajor(t0 + 3 * kProbeTile + ks);
      dev::mma_f8f6f4(d_re, are, bre, idesc, it > 0);
      dev::mma_f8f6f4(d_im, are, bim, idesc, it > 0);
      dev::mma_f8f6f4(d_re, aim, bim, idesc, 1);
      dev::mma_f8f6f4(d_im, aim, bre, idesc_neg, 1);
    }
    dev::mma_commit(dev::smem_u32(bar));
  }
  volatile int never = 0;
  if (!dev::mbar_wait(dev::smem_u32(bar), 0, &never)) {
    if (threadIdx.x == 0) atomicOr(status, dev::kStatusTimeoutOther);
  }
  dev::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    dev::tc_fence_after();
    dev::tmem_dealloc(tmem, 512);
  }
}

}  // namespace
}  // namespace ftdx

using namespace ftdx;

extern "C" ftdx_status ftdx_peak_probe(ftdx_handle h, int kind, int iters, int reps, double* tflops) {
  if (!h || !tflops || kind < 0 || kind > 3 || iters < 1 || reps < 1)
    return FTDX_ERR_INVALID_ARG;
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  const bool single = kind == 3;
  e = ensure_smem_limit(single ? reinterpret_cast<const void*>(peak_probe_single_kernel)
                               : reinterpret_cast<const void*>(peak_probe_kernel),
                        kProbeSmem);
  if (e != cudaSuccess) return cuda_fail(h, e, "probe attributes");
  // issuers: SM pairs (clusters) for kinds 0-2, SMs for kind 3
  int issuers = 0;
  if (single) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, peak_probe_single_kernel, 128,
                                                      kProbeSmem);
    if (e != cudaSuccess || per_sm < 1) return cuda_fail(h, e, "probe occupancy");
    issuers = h->sm_count;
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(h->sm_count & ~1), 1, 1);
    cfg.blockDim = dim3(128, 1, 1);
    cfg.dynamicSmemBytes = kProbeSmem;
    e = cudaOccupancyMaxActiveClusters(&issuers, peak_probe_kernel, &cfg);
    if (e != cudaSuccess || issuers < 1) return cuda_fail(h, e, "probe occupancy");
    if (issuers > h->sm_count / 2) issuers = h->sm_count / 2;
  }
  // the data kinds issue whole k-steps: 2 (kind 2) or 4 (kind 3) MMAs
  const int step = kind == 2 ? 2 : (kind == 3 ? 4 : 1);
  const int mmas = (iters + step - 1) / step * step;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaStream_t s = nullptr;
  float best = 1e30f;
  for (int r = 0; r < reps + 1; ++r) {  // the first launch warms up
    cudaEventRecord(a, s);
    if (single)
      peak_probe_single_kernel<<<issuers, 128, kProbeSmem, s>>>(mmas, h->d_status);
    else
      peak_probe_kernel<<<2 * issuers, 128, kProbeSmem, s>>>(kind, mmas, h->d_status);
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
  const double k = kind == 1 ? 64.0 : 32.0;
  const double mn = single ? 128.0 * 128.0 : 256.0 * 256.0;
  const double flop = 2.0 * mn * k * double(mmas) * double(issuers);
  *tflops = flop / (double(best) * 1e-3) / 1e12;
  return FTDX_OK;
}
