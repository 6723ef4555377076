// herk_fp8.cu -- B200 (sm_100a) correlator kernels.
//
//  * qc_to_z_kernel / fp16_to_z_kernel: promote QC int4 (or interleaved FP16)
//    voltages to the FP8 E4M3 operand Z (x rows and conjugate-permuted y
//    rows), zero-padding K to a multiple of 64.  Replaces the reference's
//    cast_int4_to_fp8_interleaved (cutlass_interface/cutlass_gemm_api.cu:1566-1623).
//  * herk_fp8_tc_kernel: persistent, warp-specialised tcgen05 HERK.  Each CTA
//    walks a list of lower-triangle tiles (128 column antennas j x 128 row
//    antennas i).  TMA feeds a 4-stage shared-memory ring; one thread issues
//    tcgen05.mma kind::f8f6f4 (M=128 x N=256 x K=32) into one of two TMEM
//    accumulators; four epilogue warps drain the other accumulator with
//    tcgen05.ld and store the packed lower triangle directly.  TMEM lane j
//    holds (Re, Im) of R_ij in columns (2i, 2i+1), so a warp's 32 lanes write
//    32 consecutive packed elements of one triangle row per store.
//    Replaces herk_direct_fp8_* (cutlass_interface/shared/herk_kernel_common.hpp:175-2768)
//    and the CUTLASS baseline + pack kernels
//    (cutlass_interface/gemm_complex_sm100/api_impl.hpp:1462-1745).
#include "herk_fp8.cuh"
#include "sm100.cuh"
#include <cuda_fp16.h>
#include <cuda_fp8.h>

namespace ftdx {
using namespace dev;

// ------------------------------------------------------------------ promotion
// Four QC bytes -> E4M3 bytes of the four Re parts and of the four Im parts.
// Sign-magnitude nibble: bit 3 sign, bits 2:0 magnitude (0..7).  E4M3 codes of
// the integers 0..7 are 00 38 40 44 48 4A 4C 4E; a byte permute indexed by the
// magnitude looks them up, the sign goes to bit 7.
__device__ __forceinline__ void qc4_to_e4m3(uint32_t w, uint32_t& re, uint32_t& im) {
  constexpr uint32_t kLo = 0x44403800u, kHi = 0x4E4C4A48u;
  const uint32_t mr = (w >> 4) & 0x07070707u;
  const uint32_t mi = w & 0x07070707u;
  uint32_t sr = mr | (mr >> 4);
  sr = (sr & 0xFFu) | ((sr >> 8) & 0xFF00u);
  uint32_t si = mi | (mi >> 4);
  si = (si & 0xFFu) | ((si >> 8) & 0xFF00u);
  re = __byte_perm(kLo, kHi, sr) | (w & 0x80808080u);
  im = __byte_perm(kLo, kHi, si) | ((w << 4) & 0x80808080u);
}

// Interleave: x = (re0, im0, re1, im1, ...), y = (im0, -re0, im1, -re1, ...).
__device__ __forceinline__ void make_xy(uint32_t re, uint32_t im, uint32_t& x0, uint32_t& x1,
                                        uint32_t& y0, uint32_t& y1) {
  const uint32_t nre = re ^ 0x80808080u;
  x0 = __byte_perm(re, im, 0x5140);
  x1 = __byte_perm(re, im, 0x7362);
  y0 = __byte_perm(im, nre, 0x5140);
  y1 = __byte_perm(im, nre, 0x7362);
}

// One thread converts 16 samples of one antenna row.
__global__ void __launch_bounds__(256) qc_to_z_kernel(const uint8_t* __restrict__ qc,
                                                      uint8_t* __restrict__ z, int64_t rows,
                                                      int K, int Kp) {
  const int chunks = Kp >> 4;
  const int64_t total = rows * chunks;
  const int64_t zpitch = 2 * int64_t(Kp);
  const bool vec = ((K & 15) == 0) && ((reinterpret_cast<uintptr_t>(qc) & 15) == 0);
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = idx / chunks;
    const int t0 = int(idx - r * chunks) << 4;
    const uint8_t* src = qc + r * K + t0;
    uint32_t w[4];
    if (vec && t0 + 16 <= K) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(src));
      w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t acc = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int t = t0 + 4 * q + b;
          const uint32_t byte = (t < K) ? uint32_t(__ldg(src + 4 * q + b)) : 0u;
          acc |= byte << (8 * b);
        }
        w[q] = acc;
      }
    }
    uint32_t x[8], y[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t re, im;
      qc4_to_e4m3(w[q], re, im);
      make_xy(re, im, x[2 * q], x[2 * q + 1], y[2 * q], y[2 * q + 1]);
    }
    uint4* dx = reinterpret_cast<uint4*>(z + (2 * r) * zpitch + 2 * t0);
    uint4* dy = reinterpret_cast<uint4*>(z + (2 * r + 1) * zpitch + 2 * t0);
    dx[0] = make_uint4(x[0], x[1], x[2], x[3]);
    dx[1] = make_uint4(x[4], x[5], x[6], x[7]);
    dy[0] = make_uint4(y[0], y[1], y[2], y[3]);
    dy[1] = make_uint4(y[4], y[5], y[6], y[7]);
  }
}

// Interleaved FP16 complex [rows][K][2] -> Z.  FP16 -> E4M3 rounds to nearest
// and saturates at +-448 with no scaling, as the reference's FP16 -> FP8 cast
// (cutlass_interface/shared/cast_kernels_common.hpp:34-37).
__device__ __forceinline__ uint32_t h2_to_e4m3x2(__half2 h) {
  return uint32_t(__nv_cvt_halfraw2_to_fp8x2(static_cast<__half2_raw>(h), __NV_SATFINITE,
                                             __NV_E4M3));
}

__global__ void __launch_bounds__(256) fp16_to_z_kernel(const __half2* __restrict__ a,
                                                        uint8_t* __restrict__ z, int64_t rows,
                                                        int K, int Kp) {
  const int chunks = Kp >> 3;  // 8 samples per thread
  const int64_t total = rows * chunks;
  const int64_t zpitch = 2 * int64_t(Kp);
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = idx / chunks;
    const int t0 = int(idx - r * chunks) << 3;
    uint32_t x[4], y[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t pr[2];
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int t = t0 + 2 * q + b;
        __half2 h = (t < K) ? a[r * K + t] : __floats2half2_rn(0.f, 0.f);
        pr[b] = h2_to_e4m3x2(h);  // low byte Re, high byte Im
      }
      x[q] = pr[0] | (pr[1] << 16);
      // y = (im, -re) per sample
      const uint32_t y0 = ((pr[0] >> 8) & 0xFFu) | (((pr[0] & 0xFFu) ^ 0x80u) << 8);
      const uint32_t y1 = ((pr[1] >> 8) & 0xFFu) | (((pr[1] & 0xFFu) ^ 0x80u) << 8);
      y[q] = y0 | (y1 << 16);
    }
    *reinterpret_cast<uint4*>(z + (2 * r) * zpitch + 2 * t0) = make_uint4(x[0], x[1], x[2], x[3]);
    *reinterpret_cast<uint4*>(z + (2 * r + 1) * zpitch + 2 * t0) =
        make_uint4(y[0], y[1], y[2], y[3]);
  }
}

// ------------------------------------------------------------------ HERK
__device__ __forceinline__ void store_elem(float* out, int64_t idx, float re, float im,
                                           float beta) {
  float2* p = reinterpret_cast<float2*>(out) + idx;
  if (beta != 0.f) {
    const float2 o = __ldcs(p);
    re += beta * o.x;
    im += beta * o.y;
  }
  __stcs(p, make_float2(re, im));
}
__device__ __forceinline__ void store_elem(__half* out, int64_t idx, float re, float im,
                                           float beta) {
  __half2* p = reinterpret_cast<__half2*>(out) + idx;
  if (beta != 0.f) {
    const float2 o = __half22float2(*p);
    re += beta * o.x;
    im += beta * o.y;
  }
  *p = __floats2half2_rn(re, im);
}

template <typename OutT>
__global__ void __launch_bounds__(kHerkThreads, 1)
    herk_fp8_tc_kernel(const __grid_constant__ CUtensorMap tmX,
                       const __grid_constant__ CUtensorMap tmZ, const HerkArgs args) {
  extern __shared__ uint8_t smem_dyn[];
  // 128 B swizzled operand tiles must start on 1024 B boundaries of the
  // shared window.
  uint8_t* smem = smem_dyn + ((1024u - (smem_u32(smem_dyn) & 1023u)) & 1023u);
  uint8_t* sA = smem;
  uint8_t* sB = smem + kStages * kABytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (kStages + s); };
  auto tfull_bar = [&](int b) { return bar0 + 8u * (2 * kStages + b); };
  auto tempty_bar = [&](int b) { return bar0 + 8u * (2 * kStages + 2 + b); };
  const uint32_t done_bar = bar0 + 8u * (2 * kStages + 4);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull_bar(b), 1);
      mbar_init(tempty_bar(b), 4);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmX);
    tma_prefetch_desc(&tmZ);
  }
  if (warp == 1) {
    tmem_alloc(smem_u32(tmem_slot), 2 * kAccCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------ TMA producer
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int issued = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
        const TileDesc td = args.tiles[t];
        const ChanDesc cd = args.chans[td.ch];
        const int32_t rowJ = int32_t(cd.row0 + int64_t(td.tj) * kBlockJ);
        const int32_t rowZ = int32_t(2 * (cd.row0 + int64_t(td.ti) * kBlockI));
        for (int kb = 0; kb < cd.kblocks; ++kb) {
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutProducer);
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(full_bar(stage), kStageBytes);
          tma_load_2d(smem_u32(sA + stage * kABytes), &tmX, kb * kKBytes, rowJ, full_bar(stage));
          tma_load_2d(smem_u32(sB + stage * kBBytes), &tmZ, kb * kKBytes, rowZ, full_bar(stage));
          ++issued;
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) {
        // Let every load still in flight land before the CTA exits.
        int s = stage;
        uint32_t ph = phase;
        for (int n = 0; n < kStages && n < issued; ++n) {
          if (--s < 0) {
            s = kStages - 1;
            ph ^= 1u;
          }
          volatile int never = 0;
          mbar_wait(full_bar(s), ph, &never);
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_f32acc(0, 0, kBlockJ, kUmmaN);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
        const ChanDesc cd = args.chans[args.tiles[t].ch];
        if (!mbar_wait(tempty_bar(acc), acc_phase ^ 1u, abort_flag)) {
          atomicOr(args.status, kStatusTimeoutMma);
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + uint32_t(acc * kAccCols);
        for (int kb = 0; kb < cd.kblocks; ++kb) {
          if (!mbar_wait(full_bar(stage), phase, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutMma);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(sA + stage * kABytes);
          const uint32_t b0 = smem_u32(sB + stage * kBBytes);
#pragma unroll
          for (int s = 0; s < kKBytes / 32; ++s) {
            mma_f8f6f4(d_tmem, sdesc_sw128_kmajor(a0 + 32 * s), sdesc_sw128_kmajor(b0 + 32 * s),
                       idesc, (kb | s) != 0);
          }
          mma_commit(empty_bar(stage));
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit(tfull_bar(acc));
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1u;
        }
      }
      // No MMA may still be writing TMEM when it is released.
      mma_commit(done_bar);
      volatile int never = 0;
      mbar_wait(done_bar, 0, &never);
    }
  } else {
    // ------------------------------------------------ epilogue (warps 2..5)
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    int acc = 0;
    uint32_t acc_phase = 0;
    OutT* out = static_cast<OutT*>(args.out);
    for (int t = blockIdx.x; t < args.num_tiles; t += gridDim.x) {
      const TileDesc td = args.tiles[t];
      const ChanDesc cd = args.chans[td.ch];
      const bool ok = __all_sync(0xffffffffu, mbar_wait(tfull_bar(acc), acc_phase, abort_flag));
      if (!ok) {
        if (lane == 0) atomicOr(args.status, kStatusTimeoutEpilogue);
        break;
      }
      tc_fence_after();
      const int n = cd.n;
      const int jw = int(td.tj) * kBlockJ + q * 32;  // first column of this warp
      const int j = jw + lane;
      const int ib = int(td.ti) * kBlockI;
      OutT* outc = out + 2 * cd.out0;
      const uint32_t tb = tmem_base + (uint32_t(q * 32) << 16) + uint32_t(acc * kAccCols);
#pragma unroll 1
      for (int c = 0; c < kUmmaN / 32; ++c) {
        const int i0 = ib + 16 * c;
        if (i0 + 15 < jw || i0 >= n) continue;  // warp-uniform: nothing to store
        uint32_t r[32];
        __syncwarp();
        tmem_ld_32x32b_x32(tb + 32u * c, r);
        tmem_wait_ld();
#pragma unroll
        for (int m = 0; m < 16; ++m) {
          const int i = i0 + m;
          if (i < n && j <= i) {
            float re = __uint_as_float(r[2 * m]) * args.alpha;
            float im = (i == j) ? 0.f : __uint_as_float(r[2 * m + 1]) * args.alpha;
            store_elem(outc, int64_t(i) * (i + 1) / 2 + j, re, im, args.beta);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty_bar(acc));
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1u;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem_base, 2 * kAccCols);
  }
}

// ------------------------------------------------------------------ launchers
static int grid_for(int64_t work, int threads, int sm_count) {
  int64_t blocks = (work + threads - 1) / threads;
  const int64_t cap = int64_t(sm_count) * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return int(blocks);
}

cudaError_t launch_qc_to_z(const uint8_t* qc, uint8_t* z, int64_t rows, int K, int Kp,
                           int sm_count, cudaStream_t s) {
  const int64_t work = rows * (Kp >> 4);
  qc_to_z_kernel<<<grid_for(work, 256, sm_count), 256, 0, s>>>(qc, z, rows, K, Kp);
  return cudaGetLastError();
}

cudaError_t launch_fp16_to_z(const void* a16, uint8_t* z, int64_t rows, int K, int Kp,
                             int sm_count, cudaStream_t s) {
  const int64_t work = rows * (Kp >> 3);
  fp16_to_z_kernel<<<grid_for(work, 256, sm_count), 256, 0, s>>>(
      static_cast<const __half2*>(a16), z, rows, K, Kp);
  return cudaGetLastError();
}

cudaError_t launch_herk_fp8(const CUtensorMap& tmX, const CUtensorMap& tmZ, const HerkArgs& a,
                            int grid, cudaStream_t s) {
  static bool attr_done[2] = {false, false};
  if (a.out_fp16) {
    if (!attr_done[1]) {
      cudaError_t e = cudaFuncSetAttribute(herk_fp8_tc_kernel<__half>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(kHerkSmem));
      if (e != cudaSuccess) return e;
      attr_done[1] = true;
    }
    herk_fp8_tc_kernel<__half><<<grid, kHerkThreads, kHerkSmem, s>>>(tmX, tmZ, a);
  } else {
    if (!attr_done[0]) {
      cudaError_t e = cudaFuncSetAttribute(herk_fp8_tc_kernel<float>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(kHerkSmem));
      if (e != cudaSuccess) return e;
      attr_done[0] = true;
    }
    herk_fp8_tc_kernel<float><<<grid, kHerkThreads, kHerkSmem, s>>>(tmX, tmZ, a);
  }
  return cudaGetLastError();
}

}  // namespace ftdx
