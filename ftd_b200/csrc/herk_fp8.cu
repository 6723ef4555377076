// herk_fp8.cu -- B200 (sm_100a) correlator kernels.
//
//  * qc_to_planes_kernel / fp16_to_planes_kernel: promote QC int4 (or
//    interleaved FP16) voltages to the FP8 E4M3 operand planes Z[Re|Im],
//    zero-padding K to a multiple of 128.  Replaces the reference's
//    cast_int4_to_fp8_interleaved (cutlass_interface/cutlass_gemm_api.cu:1566-1623).
//  * herk_fp8_tc_kernel: persistent, warp-specialised tcgen05 HERK.  Each CTA
//    walks a list of lower-triangle tiles (128 column antennas j x 128 row
//    antennas i).  TMA feeds a 3-stage ring of four 128 x 128-byte planes
//    (Re_j, Im_j, Re_i, Im_i); one thread issues four tcgen05.mma kind::f8f6f4
//    (M = N = 128, K = 32) per k-step into a Re and an Im accumulator in TMEM
//    (double-buffered); four epilogue warps drain the other accumulator with
//    tcgen05.ld and store the packed lower triangle directly.  TMEM lane j
//    holds R_ij for consecutive i in consecutive columns, so a warp's 32
//    lanes write 32 consecutive packed elements of one triangle row per store.
//    Replaces herk_direct_fp8_* (cutlass_interface/shared/herk_kernel_common.hpp:175-2768)
//    and the CUTLASS baseline + pack kernels
//    (cutlass_interface/gemm_complex_sm100/api_impl.hpp:1462-1745).
#include "herk_fp8.cuh"
#include "sm100.cuh"
#include "qc_codec.cuh"
#include <cuda_fp16.h>
#include <cuda_fp8.h>

namespace ftdx {
using namespace dev;

// ------------------------------------------------------------------ promotion
// qc4_to_e4m3: qc_codec.cuh

// One thread converts 16 samples of one antenna row.  Each block owns
// `rows_per_block` consecutive rows so that all index math is 32-bit.
// With neg_plane set a third plane receives -Re (sign bit flipped), the B
// operand of the CTA-pair kernel's partner CTA.
__global__ void __launch_bounds__(256) qc_to_planes_kernel(const uint8_t* __restrict__ qc,
                                                           uint8_t* __restrict__ z, int64_t rows,
                                                           int K, int Kp, int rows_per_block,
                                                           int neg_plane) {
  const int chunks = Kp >> 4;
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_block;
  const int64_t nrows64 = rows - r0 < rows_per_block ? rows - r0 : rows_per_block;
  const int nloc = int(nrows64) * chunks;
  const int64_t plane = rows * int64_t(Kp);
  const bool vec = ((K & 15) == 0) && ((reinterpret_cast<uintptr_t>(qc) & 15) == 0);
  for (int l = threadIdx.x; l < nloc; l += blockDim.x) {
    const int rl = l / chunks;
    const int t0 = (l - rl * chunks) << 4;
    const int64_t r = r0 + rl;
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
    uint32_t re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) qc4_to_e4m3(w[q], re[q], im[q]);
    uint8_t* dst = z + r * Kp + t0;
    *reinterpret_cast<uint4*>(dst) = make_uint4(re[0], re[1], re[2], re[3]);
    *reinterpret_cast<uint4*>(dst + plane) = make_uint4(im[0], im[1], im[2], im[3]);
    if (neg_plane) {
      constexpr uint32_t kS = 0x80808080u;
      *reinterpret_cast<uint4*>(dst + 2 * plane) =
          make_uint4(re[0] ^ kS, re[1] ^ kS, re[2] ^ kS, re[3] ^ kS);
    }
  }
}

// Signed 8-bit operand planes: as qc_to_planes_kernel with two's-complement
// integers instead of E4M3 codes (plane 2 = -Re by a per-byte negate).
__global__ void __launch_bounds__(256) qc_to_planes_s8_kernel(const uint8_t* __restrict__ qc,
                                                              uint8_t* __restrict__ z,
                                                              int64_t rows, int K, int Kp,
                                                              int rows_per_block, int neg_plane) {
  const int chunks = Kp >> 4;
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_block;
  const int64_t nrows64 = rows - r0 < rows_per_block ? rows - r0 : rows_per_block;
  const int nloc = int(nrows64) * chunks;
  const int64_t plane = rows * int64_t(Kp);
  const bool vec = ((K & 15) == 0) && ((reinterpret_cast<uintptr_t>(qc) & 15) == 0);
  for (int l = threadIdx.x; l < nloc; l += blockDim.x) {
    const int rl = l / chunks;
    const int t0 = (l - rl * chunks) << 4;
    const int64_t r = r0 + rl;
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
    uint32_t re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) qc4_to_s8(w[q], re[q], im[q]);
    uint8_t* dst = z + r * Kp + t0;
    *reinterpret_cast<uint4*>(dst) = make_uint4(re[0], re[1], re[2], re[3]);
    *reinterpret_cast<uint4*>(dst + plane) = make_uint4(im[0], im[1], im[2], im[3]);
    if (neg_plane)
      *reinterpret_cast<uint4*>(dst + 2 * plane) =
          make_uint4(__vsub4(0u, re[0]), __vsub4(0u, re[1]), __vsub4(0u, re[2]), __vsub4(0u, re[3]));
  }
}

// FP6 operand planes: as qc_to_planes_kernel, but each plane row holds Kp
// E3M2 codes packed 16 per 12 bytes (row pitch 3 Kp / 4 bytes), the global
// form of the TMA's 16 x U6 type.  Exact for QC input, 3/4 of the FP8 bytes.
__global__ void __launch_bounds__(256) qc_to_planes6_kernel(const uint8_t* __restrict__ qc,
                                                            uint8_t* __restrict__ z, int64_t rows,
                                                            int K, int Kp, int rows_per_block,
                                                            int neg_plane) {
  const int chunks = Kp >> 4;
  const int64_t pitch = int64_t(Kp) * 3 / 4;
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_block;
  const int64_t nrows64 = rows - r0 < rows_per_block ? rows - r0 : rows_per_block;
  const int nloc = int(nrows64) * chunks;
  const int64_t plane = rows * pitch;
  const bool vec = ((K & 15) == 0) && ((reinterpret_cast<uintptr_t>(qc) & 15) == 0);
  for (int l = threadIdx.x; l < nloc; l += blockDim.x) {
    const int rl = l / chunks;
    const int g = l - rl * chunks;
    const int t0 = g << 4;
    const int64_t r = r0 + rl;
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
    uint32_t re[4], im[4], pr[3], pi[3];
#pragma unroll
    for (int q = 0; q < 4; ++q) qc4_to_e3m2(w[q], re[q], im[q]);
    pack16_u6(re, pr);
    pack16_u6(im, pi);
    uint32_t* dst = reinterpret_cast<uint32_t*>(z + r * pitch + 12 * g);
    dst[0] = pr[0], dst[1] = pr[1], dst[2] = pr[2];
    uint32_t* dsti = reinterpret_cast<uint32_t*>(z + plane + r * pitch + 12 * g);
    dsti[0] = pi[0], dsti[1] = pi[1], dsti[2] = pi[2];
    if (neg_plane) {
#pragma unroll
      for (int q = 0; q < 4; ++q) re[q] ^= 0x20202020u;
      pack16_u6(re, pr);
      uint32_t* dstn = reinterpret_cast<uint32_t*>(z + 2 * plane + r * pitch + 12 * g);
      dstn[0] = pr[0], dstn[1] = pr[1], dstn[2] = pr[2];
    }
  }
}

// Plane 2 = plane 0 with every E4M3 sign flipped (-Re), for inputs whose
// promotion kernel writes two planes.  n16 = plane bytes / 16.
__global__ void __launch_bounds__(256) negate_plane_kernel(uint4* __restrict__ z, int64_t n16) {
  constexpr uint32_t kS = 0x80808080u;
  for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < n16;
       x += int64_t(gridDim.x) * blockDim.x) {
    const uint4 v = z[x];
    z[x + 2 * n16] = make_uint4(v.x ^ kS, v.y ^ kS, v.z ^ kS, v.w ^ kS);
  }
}

// Interleaved FP16 complex [rows][K][2] -> Z planes.  FP16 -> E4M3 rounds to
// nearest and saturates at +-448 with no scaling, as the reference's FP16 ->
// FP8 cast (cutlass_interface/shared/cast_kernels_common.hpp:34-37).
__device__ __forceinline__ uint32_t h2_to_e4m3x2(__half2 h) {
  return uint32_t(__nv_cvt_halfraw2_to_fp8x2(static_cast<__half2_raw>(h), __NV_SATFINITE,
                                             __NV_E4M3));
}

// With `vec` (uniform: K a multiple of 4 and the input 16-byte aligned) a
// thread's 8 samples are two 16-byte loads; otherwise, and past K, one
// sample at a time.
__global__ void __launch_bounds__(256) fp16_to_planes_kernel(const __half2* __restrict__ a,
                                                             uint8_t* __restrict__ z, int64_t rows,
                                                             int K, int Kp, int rows_per_block,
                                                             int vec) {
  const int chunks = Kp >> 3;  // 8 samples per thread
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_block;
  const int64_t nrows64 = rows - r0 < rows_per_block ? rows - r0 : rows_per_block;
  const int nloc = int(nrows64) * chunks;
  const int64_t plane = rows * int64_t(Kp);
  for (int l = threadIdx.x; l < nloc; l += blockDim.x) {
    const int rl = l / chunks;
    const int t0 = (l - rl * chunks) << 3;
    const int64_t r = r0 + rl;
    uint32_t re[2], im[2];
    __half2 hv[8];
    if (vec && t0 + 8 <= K) {
      const uint4* p4 = reinterpret_cast<const uint4*>(a + r * K + t0);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const uint4 v = __ldg(p4 + q);
        const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int b = 0; b < 4; ++b) hv[4 * q + b] = *reinterpret_cast<const __half2*>(&w4[b]);
      }
    } else {
#pragma unroll
      for (int b = 0; b < 8; ++b)
        hv[b] = (t0 + b < K) ? a[r * K + t0 + b] : __floats2half2_rn(0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      uint32_t pr[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) pr[b] = h2_to_e4m3x2(hv[4 * q + b]);  // byte 0 Re, byte 1 Im
      const uint32_t lo = pr[0] | (pr[1] << 16), hi = pr[2] | (pr[3] << 16);
      re[q] = __byte_perm(lo, hi, 0x6420);
      im[q] = __byte_perm(lo, hi, 0x7531);
    }
    uint8_t* dst = z + r * Kp + t0;
    *reinterpret_cast<uint2*>(dst) = make_uint2(re[0], re[1]);
    *reinterpret_cast<uint2*>(dst + plane) = make_uint2(im[0], im[1]);
  }
}

// Batched promotion with row gathering (flagged inputs) and per-channel K.
// Block (x, y): channel y, rows [x * rows_per_block, ...).  One thread
// converts 16 samples of one row.  neg_plane: plane 2 receives -Re too.
__global__ void __launch_bounds__(256) gather_qc_to_planes_kernel(const GatherDesc* __restrict__ gd,
                                                                  uint8_t* __restrict__ z,
                                                                  int64_t total_rows, int Kp,
                                                                  int rows_per_block,
                                                                  int neg_plane) {
  const GatherDesc g = gd[blockIdx.y];
  const int r0 = blockIdx.x * rows_per_block;
  if (r0 >= g.n) return;
  const int nrows = min(rows_per_block, g.n - r0);
  const int kpc = (g.k + kStageK - 1) / kStageK * kStageK;  // this channel's padded K
  const int chunks = kpc >> 4;
  const int64_t plane = total_rows * int64_t(Kp);
  const bool vec = ((g.lda & 15) == 0) && ((reinterpret_cast<uintptr_t>(g.a) & 15) == 0);
  for (int l = threadIdx.x; l < nrows * chunks; l += blockDim.x) {
    const int rl = l / chunks;
    const int t0 = (l - rl * chunks) << 4;
    const int r = r0 + rl;
    const int64_t src_row = g.active ? int64_t(__ldg(g.active + r)) : int64_t(r);
    const uint8_t* src = g.a + src_row * g.lda + t0;
    uint32_t w[4];
    if (vec && t0 + 16 <= g.k) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(src));
      w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t acc = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int t = t0 + 4 * q + b;
          const uint32_t byte = (t < g.k) ? uint32_t(__ldg(src + 4 * q + b)) : 0u;
          acc |= byte << (8 * b);
        }
        w[q] = acc;
      }
    }
    uint32_t re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) qc4_to_e4m3(w[q], re[q], im[q]);
    uint8_t* dst = z + (g.row0 + r) * int64_t(Kp) + t0;
    *reinterpret_cast<uint4*>(dst) = make_uint4(re[0], re[1], re[2], re[3]);
    *reinterpret_cast<uint4*>(dst + plane) = make_uint4(im[0], im[1], im[2], im[3]);
    if (neg_plane) {
      constexpr uint32_t kS = 0x80808080u;
      *reinterpret_cast<uint4*>(dst + 2 * plane) =
          make_uint4(re[0] ^ kS, re[1] ^ kS, re[2] ^ kS, re[3] ^ kS);
    }
  }
}

// ------------------------------------------------------------------ HERK
// Output element stores.  Streaming (.cs) stores: the triangle is written
// once and never re-read by this kernel.
__device__ __forceinline__ void put(float2* p, float re, float im) { __stcs(p, make_float2(re, im)); }
__device__ __forceinline__ void put(__half2* p, float re, float im) {
  *p = __floats2half2_rn(re, im);
}
__device__ __forceinline__ float2 get(const float2* p) { return __ldcs(p); }
__device__ __forceinline__ float2 get(const __half2* p) { return __half22float2(*p); }

template <typename T> struct Complex2;
template <> struct Complex2<float> { using type = float2; };
template <> struct Complex2<__half> { using type = __half2; };

// Epilogue store of one warp's 32-row chunk: lane = column j, re/im[m] hold
// element (i0 + m, j); p points at element (i0, j) of the packed triangle and
// row i+1 starts i+1 elements after row i.  `full` (warp-uniform): all 32
// rows lie below n and strictly below the diagonal (j < i), so no element
// needs a bounds check or the Im(diagonal) = 0 rule.  The fast paths cover
// the plain (C = A A^H) and scaled (alpha, per-channel scale) stores; beta and
// Kahan read the old value first.
// XEngine output formats (HerkArgs::out_format 1 / 2): element (i, j <= i)
// of R = sum_t v_i conj(v_j) is C(j, i) of C = sum_t conj(v_r) v_c, stored in
// the packed upper triangle (format 1) or the full matrix with its mirror
// C(i, j) = conj(R_ij) (format 2).  ob: this channel's output.
template <typename Out2>
__device__ __forceinline__ void store_chunk_xengine(Out2* ob, int i0, int j, int n, float sc,
                                                    int format, const uint32_t (&re)[32],
                                                    const uint32_t (&im)[32]) {
#pragma unroll
  for (int m = 0; m < 32; ++m) {
    const int i = i0 + m;
    if (i < n && j <= i) {
      const float vr = __uint_as_float(re[m]) * sc;
      const float vi = (i == j) ? 0.f : __uint_as_float(im[m]) * sc;
      if (format == 1) {
        put(ob + (int64_t(j) * n - int64_t(j) * (j - 1) / 2 + (i - j)), vr, vi);
      } else {
        put(ob + int64_t(j) * n + i, vr, vi);
        if (i != j) put(ob + int64_t(i) * n + j, vr, -vi);
      }
    }
  }
}

template <int R, typename Out2>
__device__ __forceinline__ void store_chunk(Out2* p, float2* pc, int i0, int j, int n, bool full,
                                            float sc, const HerkArgs& args,
                                            const uint32_t (&re)[R], const uint32_t (&im)[R]) {
  const bool general = args.kahan || args.beta != 0.f;
  if (full && !general) {
    if (sc == 1.f) {
#pragma unroll
      for (int m = 0; m < R; ++m) {
        put(p, __uint_as_float(re[m]), __uint_as_float(im[m]));
        p += i0 + m + 1;
      }
    } else {
#pragma unroll
      for (int m = 0; m < R; ++m) {
        put(p, __uint_as_float(re[m]) * sc, __uint_as_float(im[m]) * sc);
        p += i0 + m + 1;
      }
    }
    return;
  }
#pragma unroll
  for (int m = 0; m < R; ++m) {
    const int i = i0 + m;
    if (i < n && j <= i) {
      float vr = __uint_as_float(re[m]) * sc;
      float vi = (i == j) ? 0.f : __uint_as_float(im[m]) * sc;
      if (args.kahan) {
        // sum += v with the rounding error carried in the compensation
        const float2 sum = get(p), cmp = *pc;
        const float yr = __fsub_rn(vr, cmp.x), yi = __fsub_rn(vi, cmp.y);
        const float tr = __fadd_rn(sum.x, yr), ti = __fadd_rn(sum.y, yi);
        *pc = make_float2(__fsub_rn(__fsub_rn(tr, sum.x), yr), __fsub_rn(__fsub_rn(ti, sum.y), yi));
        vr = tr;
        vi = ti;
      } else if (args.beta != 0.f) {
        const float2 o = get(p);
        vr += args.beta * o.x;
        vi += args.beta * o.y;
      }
      put(p, vr, vi);
    }
    p += i + 1;
    if (args.kahan) pc += i + 1;
  }
}

// kFused (QC input only): tmZ maps the raw QC bytes [rows][K] instead of the
// operand planes; the producer loads raw tiles (128 rows x 128 samples, one
// byte each) into a ring of kRawStages, and four converter warps (warps 10-13)
// turn each into the E4M3 Re / Im planes of an operand stage in the 128-byte
// swizzled layout the TMA would have written, then release it to the MMA warp.
template <typename OutT, bool kFused>
__global__ void __launch_bounds__(kFused ? kFusedThreads : kHerkThreads, 1)
    herk_fp8_tc_kernel(const __grid_constant__ CUtensorMap tmZ, const HerkArgs args) {
  constexpr int kOpStages = kFused ? kFusedStages : kStages;
  constexpr int kBarCount = 2 * kOpStages + 5 + (kFused ? 2 * kRawStages : 0);
  extern __shared__ uint8_t smem_dyn[];
  // 128 B swizzled operand tiles must start on 1024 B boundaries of the
  // shared window.
  uint8_t* smem = smem_dyn + ((1024u - (smem_u32(smem_dyn) & 1023u)) & 1023u);
  // epilogue staging (kStgBytes); with kFused the raw QC ring instead
  uint8_t* stg_base = smem + kOpStages * kStageBytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(
      stg_base + (kFused ? size_t(kRawStages) * kRawStageBytes : size_t(kStgBytes)));
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kBarCount);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const uint32_t smem0 = smem_u32(smem);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (kOpStages + s); };
  auto tfull_bar = [&](int b) { return bar0 + 8u * (2 * kOpStages + b); };
  auto tempty_bar = [&](int b) { return bar0 + 8u * (2 * kOpStages + 2 + b); };
  const uint32_t done_bar = bar0 + 8u * (2 * kOpStages + 4);
  // raw ring (kFused): rfull = the TMA's bytes landed, rempty = converted
  auto rfull_bar = [&](int r) { return bar0 + 8u * (2 * kOpStages + 5 + r); };
  auto rempty_bar = [&](int r) { return bar0 + 8u * (2 * kOpStages + 5 + kRawStages + r); };
  auto raw_addr = [&](int r) {
    return smem0 + uint32_t(kOpStages * kStageBytes + r * kRawStageBytes);
  };
  // plane p of stage s: 0 = Re_j, 1 = Im_j, 2 = Re_i, 3 = Im_i
  auto plane_addr = [&](int s, int p) {
    return smem0 + uint32_t(s * kStageBytes + p * kPlaneBytes);
  };

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kOpStages; ++s) {
      mbar_init(full_bar(s), kFused ? kConvThreads : 1);  // converter threads or the TMA
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull_bar(b), 1);
      mbar_init(tempty_bar(b), kEpiWarps);
    }
    mbar_init(done_bar, 1);
    if (kFused) {
      for (int r = 0; r < kRawStages; ++r) {
        mbar_init(rfull_bar(r), 1);
        mbar_init(rempty_bar(r), kConvThreads);
      }
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) tma_prefetch_desc(&tmZ);
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
    if (kFused && lane == 0) {
      // raw QC tiles: the j block's 128 rows, then (off the diagonal) the i
      // block's, 128 bytes (samples) each; bytes past K arrive as zeros
      int r = 0;
      uint32_t rph = 0;
      int issued = 0;
      bool ok = true;
      for (TileWalk w(args.tiles, args.chans, args.num_tiles, blockIdx.x, gridDim.x);
           w.valid() && ok; w.advance()) {
        const TileDesc td = w.td;
        const ChanDesc cd = w.cd;
        const int32_t rowJ = int32_t(cd.row0 + int64_t(td.tj) * kTile);
        const int32_t rowI = int32_t(cd.row0 + int64_t(td.ti) * kTile);
        const bool diag = td.ti == td.tj;
        for (int kb = 0; kb < cd.kblocks; ++kb) {
          if (!mbar_wait(rempty_bar(r), rph ^ 1u, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutProducer);
            ok = false;
            break;
          }
          const int32_t x = (cd.kb0 + kb) * kStageK;
          mbar_arrive_expect_tx(rfull_bar(r), diag ? kPlaneBytes : 2 * kPlaneBytes);
          tma_load_2d(raw_addr(r), &tmZ, x, rowJ, rfull_bar(r));
          if (!diag) tma_load_2d(raw_addr(r) + kPlaneBytes, &tmZ, x, rowI, rfull_bar(r));
          ++issued;
          if (++r == kRawStages) {
            r = 0;
            rph ^= 1u;
          }
        }
      }
      if (!ok) {
        // Let every load still in flight land before the CTA exits.
        for (int n = 0; n < kRawStages && n < issued; ++n) {
          if (--r < 0) {
            r = kRawStages - 1;
            rph ^= 1u;
          }
          volatile int never = 0;
          if (!mbar_wait(rfull_bar(r), rph, &never)) atomicOr(args.status, kStatusTimeoutOther);
        }
      }
    } else if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int issued = 0;
      bool ok = true;
      for (TileWalk w(args.tiles, args.chans, args.num_tiles, blockIdx.x, gridDim.x);
           w.valid() && ok; w.advance()) {
        const TileDesc td = w.td;
        const ChanDesc cd = w.cd;
        // the packed-upper output format swaps the blocks: TMEM lane = larger index
        const bool swap = args.out_format == 1;
        const int32_t rowJ = int32_t(cd.row0 + int64_t(swap ? td.ti : td.tj) * kTile);
        const int32_t rowI = int32_t(cd.row0 + int64_t(swap ? td.tj : td.ti) * kTile);
        const bool diag = td.ti == td.tj;  // i block == j block: load it once
        const int nkb = cd.kblocks * args.nseg;
        for (int kb = 0; kb < nkb; ++kb) {
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutProducer);
            ok = false;
            break;
          }
          const int seg = kb / cd.kblocks;
          const int kk = kb - seg * cd.kblocks;
          const int sa = seg == 0 ? args.seg_a[0] : (seg == 1 ? args.seg_a[1] : args.seg_a[2]);
          const int sb = seg == 0 ? args.seg_b[0] : (seg == 1 ? args.seg_b[1] : args.seg_b[2]);
          const int32_t kA = (sa + cd.kb0 + kk) * kStageK, kB = (sb + cd.kb0 + kk) * kStageK;
          const bool share = diag && sa == sb;
          const uint32_t bytes = share ? 2 * kPlaneBytes : kStageBytes;  // FP8 planes
          mbar_arrive_expect_tx(full_bar(stage), args.fp6 ? bytes / 4 * 3 : bytes);
          tma_load_3d(plane_addr(stage, 0), &tmZ, kA, rowJ, 0, full_bar(stage));
          tma_load_3d(plane_addr(stage, 1), &tmZ, kA, rowJ, 1, full_bar(stage));
          if (!share) {
            tma_load_3d(plane_addr(stage, 2), &tmZ, kB, rowI, 0, full_bar(stage));
            tma_load_3d(plane_addr(stage, 3), &tmZ, kB, rowI, 1, full_bar(stage));
          }
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
          if (!mbar_wait(full_bar(s), ph, &never)) atomicOr(args.status, kStatusTimeoutOther);
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t fmt = args.fp6 ? kFmtE3M2 : kFmtE4M3;
      const uint32_t idesc = idesc_f32acc(fmt, fmt, kTile, kTile);
      const uint32_t idesc_neg = idesc_f32acc(fmt, fmt, kTile, kTile, 1);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (TileWalk w(args.tiles, args.chans, args.num_tiles, blockIdx.x, gridDim.x);
           w.valid() && ok; w.advance()) {
        const TileDesc td = w.td;
        const ChanDesc cd = w.cd;
        const bool diag = td.ti == td.tj;
        if (!mbar_wait(tempty_bar(acc), acc_phase ^ 1u, abort_flag)) {
          atomicOr(args.status, kStatusTimeoutMma);
          break;
        }
        tc_fence_after();
        const uint32_t d_re = tmem_base + uint32_t(acc * kAccCols);
        const uint32_t d_im = d_re + uint32_t(kTile);
        const int nkb = cd.kblocks * args.nseg;
        for (int kb = 0; kb < nkb; ++kb) {
          if (!mbar_wait(full_bar(stage), phase, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutMma);
            ok = false;
            break;
          }
          tc_fence_after();
          const int seg = kb / cd.kblocks;
          const int sa = seg == 0 ? args.seg_a[0] : (seg == 1 ? args.seg_a[1] : args.seg_a[2]);
          const int sb = seg == 0 ? args.seg_b[0] : (seg == 1 ? args.seg_b[1] : args.seg_b[2]);
          const int pb = (diag && sa == sb) ? 0 : 2;  // planes holding the i block
          const uint32_t are = plane_addr(stage, 0), aim = plane_addr(stage, 1);
          const uint32_t bre = plane_addr(stage, pb), bim = plane_addr(stage, pb + 1);
#pragma unroll
          for (int s = 0; s < kStageK / 32; ++s) {
            const uint64_t dare = sdesc_sw128_kmajor(are + 32 * s);
            const uint64_t daim = sdesc_sw128_kmajor(aim + 32 * s);
            const uint64_t dbre = sdesc_sw128_kmajor(bre + 32 * s);
            const uint64_t dbim = sdesc_sw128_kmajor(bim + 32 * s);
            const uint32_t first = (kb | s) != 0;
            mma_f8f6f4(d_re, dare, dbre, idesc, first);     // Re += Re_j Re_i
            mma_f8f6f4(d_im, dare, dbim, idesc, first);     // Im += Re_j Im_i
            mma_f8f6f4(d_re, daim, dbim, idesc, 1);         // Re += Im_j Im_i
            mma_f8f6f4(d_im, daim, dbre, idesc_neg, 1);     // Im -= Im_j Re_i
          }
          mma_commit(empty_bar(stage));
          if (++stage == kOpStages) {
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
      if (!mbar_wait(done_bar, 0, &never)) atomicOr(args.status, kStatusTimeoutOther);
    }
  } else if (warp < 2 + kEpiWarps) {
    // ------------------------------------------------ epilogue warps
    // Warp w may read TMEM lanes 32*(w%4)..+31 (columns j); the four warps
    // of a half own rows [64h, 64h+64) of the tile and sync on barrier 1+h.
    using Out2 = typename Complex2<OutT>::type;
    constexpr int kChunks = kTile / 32 / (kEpiWarps / 4);
    constexpr bool kBulkOut = sizeof(Out2) == 8;  // complex64 rows: 1 KB per tile row
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const uint32_t bar_id = 1u + uint32_t(half);
    const bool plain = (args.alpha == 1.f) && (args.beta == 0.f) && !args.kahan &&
                       args.chan_scale == nullptr;
    const uint32_t stg = smem_u32(stg_base) + uint32_t(half * 2 * kStgRows * kStgRowBytes);
    const bool issuer = (q == 0) && (lane < kStgRows);  // issues one row copy per sub-chunk
    int acc = 0;
    uint32_t acc_phase = 0;
    Out2* out = static_cast<Out2*>(args.out);
    for (TileWalk w(args.tiles, args.chans, args.num_tiles, blockIdx.x, gridDim.x); w.valid();
         w.advance()) {
      const TileDesc td = w.td;
      const ChanDesc cd = w.cd;
      const bool ok = bar_red_and(bar_id, 128, mbar_wait(tfull_bar(acc), acc_phase, abort_flag));
      if (!ok) {
        if (lane == 0) atomicOr(args.status, kStatusTimeoutEpilogue);
        break;
      }
      tc_fence_after();
      const int n = cd.n;
      const int j0 = int(td.tj) * kTile;
      const int jw = j0 + q * 32;  // first column of this warp
      const int j = jw + lane;
      const int ib = int(td.ti) * kTile;
      const uint32_t tb = tmem_base + (uint32_t(q * 32) << 16) + uint32_t(acc * kAccCols);
      Out2* outc = cd.out_ptr ? reinterpret_cast<Out2*>(cd.out_ptr) : out + cd.out0;
      if (!kFused && kBulkOut && args.bulk_store && plain && td.ti != td.tj && ib + kTile <= n) {
        // Interior tile: stage kStgRows row segments (128 consecutive packed
        // elements each) in shared memory, then one bulk copy per row.  A
        // row whose global start is 8 mod 16 keeps that phase in shared
        // memory; its first and last elements are stored directly.
#pragma unroll 1
        for (int sc = 0; sc < (kTile / 2) / kStgRows; ++sc) {
          const int is = ib + half * (kTile / 2) + sc * kStgRows;
          const uint32_t col = uint32_t(half * (kTile / 2) + sc * kStgRows);
          uint32_t re[kStgRows], im[kStgRows];
          __syncwarp();
          tmem_ld_32x32b_x8(tb + col, re);
          tmem_ld_32x32b_x8(tb + uint32_t(kTile) + col, im);
          tmem_wait_ld();
          const uint32_t buf = stg + uint32_t((sc & 1) * kStgRows * kStgRowBytes);
#pragma unroll
          for (int m = 0; m < kStgRows; ++m) {
            const int i = is + m;
            Out2* g = outc + int64_t(i) * (i + 1) / 2 + j0;
            const uint32_t ph = uint32_t(reinterpret_cast<uintptr_t>(g) & 8u);
            st_shared_v2(buf + uint32_t(m * kStgRowBytes) + ph + 8u * uint32_t(q * 32 + lane),
                         re[m], im[m]);
            if (ph && ((q == 0 && lane == 0) || (q == 3 && lane == 31)))
              put(outc + int64_t(i) * (i + 1) / 2 + j, __uint_as_float(re[m]),
                  __uint_as_float(im[m]));
          }
          fence_proxy_async_smem();
          named_bar_sync(bar_id, 128);
          if (issuer) {
            const int i = is + lane;
            Out2* g = outc + int64_t(i) * (i + 1) / 2 + j0;
            const bool odd = (reinterpret_cast<uintptr_t>(g) & 8u) != 0;
            const uint32_t src = buf + uint32_t(lane * kStgRowBytes) + (odd ? 16u : 0u);
            bulk_store(odd ? static_cast<void*>(g + 1) : static_cast<void*>(g), src,
                       odd ? uint32_t((kTile - 2) * 8) : uint32_t(kTile * 8));
            bulk_commit();
            bulk_wait_read<1>();  // the other buffer is free again
          }
          named_bar_sync(bar_id, 128);
        }
      } else if (!kFused && args.out_format == 1) {
        // Packed upper triangle, row-major (the XEngine's format): the producer
        // swapped the blocks, so TMEM lane = column c (the i block) and TMEM
        // column = row r (the j block), and the accumulator holds
        // sum_t v_r conj(v_c) = conj(C(r, c)).  A warp stores 32 consecutive
        // c of one row r.
        const float sc = args.alpha * (args.chan_scale ? args.chan_scale[td.ch] : 1.f);
        const int cw = ib + q * 32;  // this warp's first column
        const int c = cw + lane;
#pragma unroll 1
        for (int cc = 0; cc < kChunks; ++cc) {
          const int ch = half * kChunks + cc;
          const int r0 = j0 + 32 * ch;
          if (r0 > cw + 31 || cw >= n) continue;  // warp-uniform: nothing to store
          uint32_t re[32], im[32];
          __syncwarp();
          tmem_ld_32x32b_x32(tb + 32u * ch, re);
          tmem_ld_32x32b_x32(tb + uint32_t(kTile) + 32u * ch, im);
          tmem_wait_ld();
          if (r0 + 31 < cw && cw + 31 < n) {
            // every element strictly above the diagonal and inside n: row
            // r + 1 starts n - r - 1 elements after element (r, c)'s row start
            Out2* p = outc + (int64_t(r0) * n - int64_t(r0) * (r0 - 1) / 2 + (c - r0));
#pragma unroll
            for (int m = 0; m < 32; ++m) {
              put(p, __uint_as_float(re[m]) * sc, -__uint_as_float(im[m]) * sc);
              p += n - (r0 + m) - 1;
            }
            continue;
          }
#pragma unroll
          for (int m = 0; m < 32; ++m) {
            const int r = r0 + m;
            if (c < n && r <= c) {
              const float vr = __uint_as_float(re[m]) * sc;
              const float vi = (r == c) ? 0.f : -__uint_as_float(im[m]) * sc;
              put(outc + (int64_t(r) * n - int64_t(r) * (r - 1) / 2 + (c - r)), vr, vi);
            }
          }
        }
      } else {
        const float sc = args.alpha * (args.chan_scale ? args.chan_scale[td.ch] : 1.f);
#pragma unroll 1
        for (int cc = 0; cc < kChunks; ++cc) {
          const int c = half * kChunks + cc;
          const int i0 = ib + 32 * c;
          if (i0 + 31 < jw || i0 >= n) continue;  // warp-uniform: nothing to store
          if constexpr (kFused) {
            // 16 rows at a time: the fused kernel's 448 threads get 128 registers
#pragma unroll 1
            for (int hr = 0; hr < 2; ++hr) {
              const int i0h = i0 + 16 * hr;
              if (i0h + 15 < jw || i0h >= n) continue;  // warp-uniform
              uint32_t re[16], im[16];
              __syncwarp();
              tmem_ld_32x32b_x16(tb + 32u * c + 16u * hr, re);
              tmem_ld_32x32b_x16(tb + uint32_t(kTile) + 32u * c + 16u * hr, im);
              tmem_wait_ld();
              const int64_t e0 = int64_t(i0h) * (i0h + 1) / 2 + j;
              float2* pc = args.kahan ? static_cast<float2*>(args.out2) + cd.out0 + e0 : nullptr;
              store_chunk(outc + e0, pc, i0h, j, n, i0h + 15 < n && jw + 31 < i0h, sc, args, re,
                          im);
            }
            continue;
          }
          uint32_t re[32], im[32];
          __syncwarp();
          tmem_ld_32x32b_x32(tb + 32u * c, re);
          tmem_ld_32x32b_x32(tb + uint32_t(kTile) + 32u * c, im);
          tmem_wait_ld();
          if (args.out_format != 0) {
            Out2* ob = args.out_format == 2 ? out + int64_t(td.ch) * n * n : outc;
            store_chunk_xengine(ob, i0, j, n, sc, args.out_format, re, im);
            continue;
          }
          // element (i, j) lives at i(i+1)/2 + j; row i+1 starts i+1 later
          const int64_t e0 = int64_t(i0) * (i0 + 1) / 2 + j;
          // compensation buffer: same layout as the output (uniform calls only)
          float2* pc = args.kahan ? static_cast<float2*>(args.out2) + cd.out0 + e0 : nullptr;
          store_chunk(outc + e0, pc, i0, j, n, i0 + 31 < n && jw + 31 < i0, sc, args, re, im);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_relaxed(tempty_bar(acc));
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1u;
      }
    }
    if (issuer) bulk_wait<0>();  // bulk stores complete before the CTA exits
  } else if (kFused) {
    // ------------------------------------------------ converter warps (kFused)
    // Per stage: 2048 16-byte chunks (1024 on the diagonal).  Chunk
    // q * 128 + ct (q < 16) is row q * 16 + (ct >> 3) (rows 128-255 = the i
    // block) and 16-byte column ct & 7; a warp's load covers 4 whole raw rows.
    // In the 128-byte swizzled layout, column c of row r sits at
    // r * 128 + ((c ^ (r & 7)) << 4) of its plane; r & 7 = (ct >> 3) & 7 for
    // every q, so each chunk's source and destination are this thread's base
    // plus a constant.  All loads of a stage are issued before any convert.
    const int ct = threadIdx.x - 32 * (2 + kEpiWarps);
    const int src_t = 16 * ct;
    const int dst_t = (ct >> 3) * 128 + (((ct & 7) ^ ((ct >> 3) & 7)) << 4);
    int r = 0, stage = 0;
    uint32_t rph = 0, phase = 0;
    bool ok = true;
    for (TileWalk w(args.tiles, args.chans, args.num_tiles, blockIdx.x, gridDim.x);
         w.valid() && ok; w.advance()) {
      const bool diag = w.td.ti == w.td.tj;  // i block == j block: 8 chunks each
      for (int kb = 0; kb < w.cd.kblocks; ++kb) {
        if (!mbar_wait(rfull_bar(r), rph, abort_flag) ||
            !mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag)) {
          atomicOr(args.status, kStatusTimeoutOther);
          ok = false;
          break;
        }
        const uint8_t* src = smem + (raw_addr(r) - smem0) + src_t;
        uint8_t* dst = smem + (plane_addr(stage, 0) - smem0) + dst_t;
        // two halves of 8 chunks (the j block's rows, then the i block's)
#pragma unroll
        for (int hb = 0; hb < 2; ++hb) {
          if (hb == 1 && diag) break;
          uint4 v[8];
#pragma unroll
          for (int q = 0; q < 8; ++q)
            v[q] = *reinterpret_cast<const uint4*>(src + (hb * 8 + q) * 2048);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            uint4 re, im;
            qc4_to_e4m3(v[q].x, re.x, im.x);
            qc4_to_e4m3(v[q].y, re.y, im.y);
            qc4_to_e4m3(v[q].z, re.z, im.z);
            qc4_to_e4m3(v[q].w, re.w, im.w);
            // rows 0-127: planes 0 / 1 (Re_j / Im_j); 128-255: planes 2 / 3
            const int off = q * 2048 + hb * 2 * kPlaneBytes;
            *reinterpret_cast<uint4*>(dst + off) = re;
            *reinterpret_cast<uint4*>(dst + off + kPlaneBytes) = im;
          }
        }
        mbar_arrive(rempty_bar(r));  // every raw chunk has been read
        fence_proxy_async_smem();  // the planes are read by the tensor core
        mbar_arrive(full_bar(stage));
        if (++r == kRawStages) {
          r = 0;
          rph ^= 1u;
        }
        if (++stage == kOpStages) {
          stage = 0;
          phase ^= 1u;
        }
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

// ------------------------------------------------------------------ CTA-pair kernel
// Same computation with tcgen05 cta_group::2 MMAs of M = 256, N = 256 over a
// pair of CTAs (a 2-CTA cluster): tile = 256 column inputs j (128 per CTA,
// TMEM lane = j) x 128 row inputs i.  The N = 256 columns of one MMA are the
// Re and Im halves of the accumulator; the B operand's first 128 rows come
// from the leader CTA's shared memory and the last 128 from the partner's:
//   MMA 1: A = Re_j, B = [Re_i | Im_i]   -> Re += Re_j Re_i, Im += Re_j Im_i
//   MMA 2: A = Im_j, B = [Im_i | -Re_i]  -> Re += Im_j Im_i, Im -= Im_j Re_i
// so the leader loads (Re_i, Im_i) and the partner (Im_i, -Re_i), the third
// operand plane holding -Re.  Two MMAs per 32 samples instead of four of
// N = 128: each MMA reads half as many operand bytes per multiply-add from
// shared memory, which bounds the single-CTA kernel.  The leader CTA (rank 0)
// owns the full barriers (the partner's loads count their bytes there) and
// issues the MMAs; each commit arrives on the matching barrier of both CTAs
// (one multicast commit);
// both CTAs' epilogue warps release an accumulator on the leader's barrier.
constexpr int kPairPlane = 128 * kStageK;  // 16 KB: 128 rows of 128 samples
constexpr int kPairStageBytes = 4 * kPairPlane;
constexpr int kPairStages = 3;
// the epilogue area: staging for the bulk store mode
constexpr size_t kPairSmem = 1024 + size_t(kPairStages) * kPairStageBytes + kStgBytes + 256;
static_assert(kPairSmem <= 232448, "shared memory per CTA");

template <typename OutT>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kHerkThreads, 1)
    herk_fp8_pair_kernel(const __grid_constant__ CUtensorMap tmZ, const HerkArgs args) {
  extern __shared__ uint8_t smem_dyn[];
  uint8_t* smem = smem_dyn + ((1024u - (smem_u32(smem_dyn) & 1023u)) & 1023u);
  uint8_t* stg_base = smem + kPairStages * kPairStageBytes;  // epilogue staging (kStgBytes)
  uint64_t* bars = reinterpret_cast<uint64_t*>(stg_base + kStgBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kPairStages + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const uint32_t smem0 = smem_u32(smem);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (kPairStages + s); };
  auto tfull_bar = [&](int b) { return bar0 + 8u * (2 * kPairStages + b); };
  auto tempty_bar = [&](int b) { return bar0 + 8u * (2 * kPairStages + 2 + b); };
  const uint32_t done_bar = bar0 + 8u * (2 * kPairStages + 4);
  // planes of stage s: Re_j, Im_j, then the B halves X (MMA 1) and Y (MMA 2)
  auto plane = [&](int s, int p) { return smem0 + uint32_t(s * kPairStageBytes + p * kPairPlane); };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const int pair = int(blockIdx.x >> 1), npairs = int(gridDim.x >> 1);

  if (threadIdx.x == 0) {
    for (int s = 0; s < kPairStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull_bar(b), 1);
      mbar_init(tempty_bar(b), 2 * kEpiWarps);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmZ);
  }
  if (warp == 1) {
    tmem_alloc_pair(smem_u32(tmem_slot), 2 * kAccCols);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // both CTAs' barriers exist before any cross-CTA signal
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------ TMA producer (both CTAs)
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      for (TileWalk w(args.tiles, args.chans, args.num_tiles, pair, npairs); w.valid();
           w.advance()) {
        const TileDesc td = w.td;
        const ChanDesc cd = w.cd;
        const int32_t rowJ = int32_t(cd.row0 + int64_t(td.tj) * 256 + 128 * rank);
        const int32_t rowI = int32_t(cd.row0 + int64_t(td.ti) * kTile);
        const int32_t pX = int32_t(rank), pY = int32_t(rank) + 1;  // leader: Re, Im; partner: Im, -Re
        const int nkb = cd.kblocks * args.nseg;
        bool ok = true;
        for (int kb = 0; kb < nkb; ++kb) {
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutProducer);
            ok = false;
            break;
          }
          const int seg = kb / cd.kblocks;
          const int kk = kb - seg * cd.kblocks;
          const int sa = seg == 0 ? args.seg_a[0] : (seg == 1 ? args.seg_a[1] : args.seg_a[2]);
          const int sb = seg == 0 ? args.seg_b[0] : (seg == 1 ? args.seg_b[1] : args.seg_b[2]);
          const int32_t kA = (sa + cd.kb0 + kk) * kStageK, kB = (sb + cd.kb0 + kk) * kStageK;
          if (leader)  // both CTAs' loads; packed FP6 planes deliver 3/4 of the bytes
            mbar_arrive_expect_tx(full_bar(stage), args.fp6 ? 2 * kPairStageBytes / 4 * 3
                                                            : 2 * kPairStageBytes);
          const uint32_t fb = map_shared(full_bar(stage), 0);
          tma_load_3d_pair(plane(stage, 0), &tmZ, kA, rowJ, 0, fb);
          tma_load_3d_pair(plane(stage, 1), &tmZ, kA, rowJ, 1, fb);
          tma_load_3d_pair(plane(stage, 2), &tmZ, kB, rowI, pX, fb);
          tma_load_3d_pair(plane(stage, 3), &tmZ, kB, rowI, pY, fb);
          if (++stage == kPairStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------ MMA issuer (leader CTA)
    if (lane == 0 && leader) {
      const uint32_t fmt = args.fp6 ? kFmtE3M2 : kFmtE4M3;
      const uint32_t idesc =
          args.s8 ? idesc_s32acc_s8(256, 2 * kTile) : idesc_f32acc(fmt, fmt, 256, 2 * kTile);
      int stage = 0, acc = 0;
      uint32_t phase = 0, acc_phase = 0;
      bool ok = true;
      for (TileWalk w(args.tiles, args.chans, args.num_tiles, pair, npairs); w.valid() && ok;
           w.advance()) {
        const ChanDesc cd = w.cd;
        if (!mbar_wait(tempty_bar(acc), acc_phase ^ 1u, abort_flag)) {
          atomicOr(args.status, kStatusTimeoutMma);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + uint32_t(acc * kAccCols);  // Re | Im columns
        const int nkb = cd.kblocks * args.nseg;
        for (int kb = 0; kb < nkb; ++kb) {
          if (!mbar_wait(full_bar(stage), phase, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutMma);
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int s = 0; s < kStageK / 32; ++s) {
            const uint64_t dare = sdesc_sw128_kmajor(plane(stage, 0) + 32 * s);
            const uint64_t daim = sdesc_sw128_kmajor(plane(stage, 1) + 32 * s);
            const uint64_t dbx = sdesc_sw128_kmajor(plane(stage, 2) + 32 * s);
            const uint64_t dby = sdesc_sw128_kmajor(plane(stage, 3) + 32 * s);
            if (args.s8) {
              mma_i8_pair(d, dare, dbx, idesc, (kb | s) != 0);
              mma_i8_pair(d, daim, dby, idesc, 1);
            } else {
              mma_f8f6f4_pair(d, dare, dbx, idesc, (kb | s) != 0);
              mma_f8f6f4_pair(d, daim, dby, idesc, 1);
            }
          }
          mma_commit_pair_both(empty_bar(stage));
          if (++stage == kPairStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
        if (!ok) break;
        mma_commit_pair_both(tfull_bar(acc));
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1u;
        }
      }
      mma_commit_pair(done_bar);
      volatile int never = 0;
      if (!mbar_wait(done_bar, 0, &never)) atomicOr(args.status, kStatusTimeoutOther);
    }
  } else {
    // ------------------------------------------------ epilogue (both CTAs)
    using Out2 = typename Complex2<OutT>::type;
    constexpr int kChunks = kTile / 32 / (kEpiWarps / 4);
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    int acc = 0;
    uint32_t acc_phase = 0;
    Out2* out = static_cast<Out2*>(args.out);
    const uint32_t bar_id = 1u + uint32_t(half);
    for (TileWalk w(args.tiles, args.chans, args.num_tiles, pair, npairs); w.valid();
         w.advance()) {
      const TileDesc td = w.td;
      const ChanDesc cd = w.cd;
      // the four warps of a half agree, so none is left alone at a named barrier
      const bool ok = bar_red_and(bar_id, 128, mbar_wait(tfull_bar(acc), acc_phase, abort_flag));
      if (!ok) {
        if (lane == 0) atomicOr(args.status, kStatusTimeoutEpilogue);
        break;
      }
      tc_fence_after();
      const int n = cd.n;
      const int jw = int(td.tj) * 256 + 128 * int(rank) + q * 32;
      const int j = jw + lane;
      const int ib = int(td.ti) * kTile;
      Out2* outc = cd.out_ptr ? reinterpret_cast<Out2*>(cd.out_ptr) : out + cd.out0;
      const uint32_t tb = tmem_base + (uint32_t(q * 32) << 16) + uint32_t(acc * kAccCols);
      const float sc = args.alpha * (args.chan_scale ? args.chan_scale[td.ch] : 1.f);
      const int jt0 = jw - q * 32;  // first of this CTA's 128 columns
      bool bulk_tile = false;
      if constexpr (sizeof(Out2) == 8) {
        bulk_tile = args.bulk_store && args.out_format == 0 && args.alpha == 1.f &&
                    args.beta == 0.f && !args.kahan && args.chan_scale == nullptr &&
                    jt0 + 127 < ib && ib + kTile <= n;
      }
      if (args.out_format == 1) {
        // Packed upper triangle, row-major (the XEngine's format): the plan's
        // tiles put column inputs c on the TMEM lanes (tj over 256) and row
        // inputs r on the TMEM columns (ti over 128), so the accumulator
        // holds sum_t v_r conj(v_c) = conj(C(r, c)).  A warp stores 32
        // consecutive c of one row r.
        const int c = j;
#pragma unroll 1
        for (int cc = 0; cc < kChunks; ++cc) {
          const int k = half * kChunks + cc;
          const int r0 = ib + 32 * k;
          if (r0 > jw + 31 || jw >= n) continue;  // warp-uniform: nothing to store
          uint32_t re[32], im[32];
          __syncwarp();
          tmem_ld_32x32b_x32(tb + 32u * k, re);
          tmem_ld_32x32b_x32(tb + uint32_t(kTile) + 32u * k, im);
          tmem_wait_ld();
          if (args.s8) {  // exact S32 sums -> FP32
#pragma unroll
            for (int m = 0; m < 32; ++m) {
              re[m] = __float_as_uint(float(int32_t(re[m])));
              im[m] = __float_as_uint(float(int32_t(im[m])));
            }
          }
          if (r0 + 31 < jw && jw + 31 < n) {
            // every element strictly above the diagonal and inside n: row
            // r + 1 starts n - r - 1 elements after element (r, c)'s row start
            Out2* p = outc + (int64_t(r0) * n - int64_t(r0) * (r0 - 1) / 2 + (c - r0));
#pragma unroll
            for (int m = 0; m < 32; ++m) {
              put(p, __uint_as_float(re[m]) * sc, -__uint_as_float(im[m]) * sc);
              p += n - (r0 + m) - 1;
            }
            continue;
          }
#pragma unroll
          for (int m = 0; m < 32; ++m) {
            const int r = r0 + m;
            if (c < n && r <= c) {
              const float vr = __uint_as_float(re[m]) * sc;
              const float vi = (r == c) ? 0.f : -__uint_as_float(im[m]) * sc;
              put(outc + (int64_t(r) * n - int64_t(r) * (r - 1) / 2 + (c - r)), vr, vi);
            }
          }
        }
      }
      if (bulk_tile) {
        // Interior tile, as the single-CTA kernel's bulk mode: 8 rows at a
        // time staged in shared memory (keeping each row's 16-byte phase),
        // one bulk copy per row; a row starting 8 mod 16 stores its first
        // and last element directly.
        const uint32_t stg = smem_u32(stg_base) + uint32_t(half * 2 * kStgRows * kStgRowBytes);
        const bool issuer = (q == 0) && (lane < kStgRows);
#pragma unroll 1
        for (int sub = 0; sub < (kTile / 2) / kStgRows; ++sub) {
          const int is = ib + half * (kTile / 2) + sub * kStgRows;
          const uint32_t col = uint32_t(half * (kTile / 2) + sub * kStgRows);
          uint32_t re[kStgRows], im[kStgRows];
          __syncwarp();
          tmem_ld_32x32b_x8(tb + col, re);
          tmem_ld_32x32b_x8(tb + uint32_t(kTile) + col, im);
          tmem_wait_ld();
          if (args.s8) {  // exact S32 sums -> FP32
#pragma unroll
            for (int m = 0; m < kStgRows; ++m) {
              re[m] = __float_as_uint(float(int32_t(re[m])));
              im[m] = __float_as_uint(float(int32_t(im[m])));
            }
          }
          const uint32_t buf = stg + uint32_t((sub & 1) * kStgRows * kStgRowBytes);
#pragma unroll
          for (int m = 0; m < kStgRows; ++m) {
            const int i = is + m;
            Out2* g = outc + int64_t(i) * (i + 1) / 2 + jt0;
            const uint32_t ph = uint32_t(reinterpret_cast<uintptr_t>(g) & 8u);
            st_shared_v2(buf + uint32_t(m * kStgRowBytes) + ph + 8u * uint32_t(q * 32 + lane),
                         re[m], im[m]);
            if (ph && ((q == 0 && lane == 0) || (q == 3 && lane == 31)))
              put(outc + int64_t(i) * (i + 1) / 2 + j, __uint_as_float(re[m]),
                  __uint_as_float(im[m]));
          }
          fence_proxy_async_smem();
          named_bar_sync(bar_id, 128);
          if (issuer) {
            const int i = is + lane;
            Out2* g = outc + int64_t(i) * (i + 1) / 2 + jt0;
            const bool odd = (reinterpret_cast<uintptr_t>(g) & 8u) != 0;
            const uint32_t src = buf + uint32_t(lane * kStgRowBytes) + (odd ? 16u : 0u);
            bulk_store(odd ? static_cast<void*>(g + 1) : static_cast<void*>(g), src,
                       odd ? uint32_t((kTile - 2) * 8) : uint32_t(kTile * 8));
            bulk_commit();
            bulk_wait_read<1>();  // the other buffer is free again
          }
          named_bar_sync(bar_id, 128);
        }
      }
#pragma unroll 1
      for (int cc = 0; cc < kChunks && !bulk_tile && args.out_format != 1; ++cc) {
        const int c = half * kChunks + cc;
        const int i0 = ib + 32 * c;
        if (i0 + 31 < jw || i0 >= n) continue;  // warp-uniform: nothing to store
        uint32_t re[32], im[32];
        __syncwarp();
        tmem_ld_32x32b_x32(tb + 32u * c, re);
        tmem_ld_32x32b_x32(tb + uint32_t(kTile) + 32u * c, im);
        tmem_wait_ld();
        if (args.s8) {  // exact S32 sums -> FP32
#pragma unroll
          for (int m = 0; m < 32; ++m) {
            re[m] = __float_as_uint(float(int32_t(re[m])));
            im[m] = __float_as_uint(float(int32_t(im[m])));
          }
        }
        if (args.out_format == 2) {  // the XEngine's full Hermitian matrix
          store_chunk_xengine(out + int64_t(td.ch) * n * n, i0, j, n, sc, 2, re, im);
          continue;
        }
        const int64_t e0 = int64_t(i0) * (i0 + 1) / 2 + j;
        float2* pc = args.kahan ? static_cast<float2*>(args.out2) + cd.out0 + e0 : nullptr;
        store_chunk(outc + e0, pc, i0, j, n, i0 + 31 < n && jw + 31 < i0, sc, args, re, im);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster_relaxed(map_shared(tempty_bar(acc), 0));
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1u;
      }
    }
    if (q == 0 && lane < kStgRows) bulk_wait<0>();  // bulk stores complete before the CTA exits
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // neither CTA leaves while the other may still signal it
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, 2 * kAccCols);
  }
}

// ------------------------------------------------------------------ launchers
static int rows_per_block(int chunks) {
  int r = 8192 / (chunks > 0 ? chunks : 1);
  return r < 1 ? 1 : r;
}

cudaError_t launch_qc_to_planes(const uint8_t* qc, uint8_t* z, int64_t rows, int K, int Kp,
                                cudaStream_t s, bool neg_plane) {
  const int rpb = rows_per_block(Kp >> 4);
  const int64_t blocks = (rows + rpb - 1) / rpb;
  qc_to_planes_kernel<<<unsigned(blocks), 256, 0, s>>>(qc, z, rows, K, Kp, rpb, neg_plane ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_qc_to_planes_s8(const uint8_t* qc, uint8_t* z, int64_t rows, int K, int Kp,
                                   cudaStream_t s, bool neg_plane) {
  const int rpb = rows_per_block(Kp >> 4);
  const int64_t blocks = (rows + rpb - 1) / rpb;
  qc_to_planes_s8_kernel<<<unsigned(blocks), 256, 0, s>>>(qc, z, rows, K, Kp, rpb,
                                                           neg_plane ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_qc_to_planes6(const uint8_t* qc, uint8_t* z, int64_t rows, int K, int Kp,
                                 cudaStream_t s, bool neg_plane) {
  const int rpb = rows_per_block(Kp >> 4);
  const int64_t blocks = (rows + rpb - 1) / rpb;
  qc_to_planes6_kernel<<<unsigned(blocks), 256, 0, s>>>(qc, z, rows, K, Kp, rpb,
                                                         neg_plane ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_negate_plane(uint8_t* z, int64_t plane_bytes, int sm_count, cudaStream_t s) {
  const int64_t n16 = plane_bytes / 16;
  int64_t blocks = (n16 + 255) / 256;
  if (blocks > int64_t(sm_count) * 8) blocks = int64_t(sm_count) * 8;
  if (blocks < 1) blocks = 1;
  negate_plane_kernel<<<unsigned(blocks), 256, 0, s>>>(reinterpret_cast<uint4*>(z), n16);
  return cudaGetLastError();
}

cudaError_t launch_fp16_to_planes(const void* a16, uint8_t* z, int64_t rows, int K, int Kp,
                                  cudaStream_t s) {
  const int rpb = rows_per_block(Kp >> 3);
  const int64_t blocks = (rows + rpb - 1) / rpb;
  fp16_to_planes_kernel<<<unsigned(blocks), 256, 0, s>>>(
      static_cast<const __half2*>(a16), z, rows, K, Kp, rpb,
      (K % 4 == 0 && (reinterpret_cast<uintptr_t>(a16) & 15) == 0) ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_gather_qc_to_planes(const GatherDesc* g, int nch, int max_n, uint8_t* z,
                                       int64_t total_rows, int Kp, cudaStream_t s, int neg_plane) {
  const int rpb = rows_per_block(Kp >> 4);
  const dim3 grid(unsigned((max_n + rpb - 1) / rpb), unsigned(nch));
  gather_qc_to_planes_kernel<<<grid, 256, 0, s>>>(g, z, total_rows, Kp, rpb, neg_plane);
  return cudaGetLastError();
}

template <typename OutT, bool kFused>
static cudaError_t launch_herk_t(const CUtensorMap& tmZ, const HerkArgs& a, int grid,
                                 cudaStream_t s) {
  constexpr size_t smem = kFused ? kFusedSmem : kHerkSmem;
  constexpr int threads = kFused ? kFusedThreads : kHerkThreads;
  cudaError_t e =
      ensure_smem_limit(reinterpret_cast<const void*>(herk_fp8_tc_kernel<OutT, kFused>), smem);
  if (e != cudaSuccess) return e;
  herk_fp8_tc_kernel<OutT, kFused><<<grid, threads, smem, s>>>(tmZ, a);
  return cudaGetLastError();
}

template <typename OutT>
static cudaError_t pair_attributes() {
  return ensure_smem_limit(reinterpret_cast<const void*>(herk_fp8_pair_kernel<OutT>), kPairSmem);
}

template <typename OutT>
static cudaError_t launch_pair_t(const CUtensorMap& tmZ, const HerkArgs& a, int grid,
                                 cudaStream_t s) {
  cudaError_t e = pair_attributes<OutT>();
  if (e != cudaSuccess) return e;
  herk_fp8_pair_kernel<OutT><<<grid, kHerkThreads, kPairSmem, s>>>(tmZ, a);
  return cudaGetLastError();
}

cudaError_t herk_fp8_pair_max_clusters(int sm_count, int* clusters) {
  cudaError_t e = pair_attributes<float>();
  if (e == cudaSuccess) e = pair_attributes<__half>();
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(sm_count & ~1), 1, 1);
  cfg.blockDim = dim3(kHerkThreads, 1, 1);
  cfg.dynamicSmemBytes = kPairSmem;
  int nf = 0, nh = 0;
  e = cudaOccupancyMaxActiveClusters(&nf, herk_fp8_pair_kernel<float>, &cfg);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&nh, herk_fp8_pair_kernel<__half>, &cfg);
  *clusters = nf < nh ? nf : nh;
  return e;
}

cudaError_t launch_herk_fp8_pair(const CUtensorMap& tmZ, const HerkArgs& a, int grid,
                                 cudaStream_t s) {
  if (grid < 2 || (grid & 1)) return cudaErrorInvalidConfiguration;
  return a.out_fp16 ? launch_pair_t<__half>(tmZ, a, grid, s) : launch_pair_t<float>(tmZ, a, grid, s);
}

// Split-K: the correlator wrote `splits` partial triangles per channel
// (ws[c*splits + s][P]); C = alpha * cs_c * sum_s partial_s + beta * C.  The
// partials of integer inputs are exact integers, so the sum is too.
template <typename Out2>
__global__ void __launch_bounds__(256) split_reduce_kernel(const float2* __restrict__ ws,
                                                           Out2* __restrict__ out, int64_t P,
                                                           int batch, int splits, float alpha,
                                                           float beta,
                                                           const float* __restrict__ chan_scale) {
  const int64_t total = int64_t(batch) * P;
  for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < total;
       x += int64_t(gridDim.x) * blockDim.x) {
    const int64_t c = x / P, p = x - c * P;
    const float2* w = ws + c * splits * P + p;
    float re = 0.f, im = 0.f;
    for (int s = 0; s < splits; ++s) {
      const float2 v = __ldcs(w + int64_t(s) * P);
      re += v.x;
      im += v.y;
    }
    const float sc = alpha * (chan_scale ? chan_scale[c] : 1.f);
    re *= sc;
    im *= sc;
    if (beta != 0.f) {
      const float2 o = get(out + x);
      re += beta * o.x;
      im += beta * o.y;
    }
    put(out + x, re, im);
  }
}

cudaError_t launch_split_reduce(const float2* ws, void* out, int out_fp16, int64_t P, int batch,
                                int splits, float alpha, float beta, const float* chan_scale,
                                int sm_count, cudaStream_t s) {
  const int64_t total = int64_t(batch) * P;
  int64_t blocks = (total + 255) / 256;
  if (blocks > int64_t(sm_count) * 16) blocks = int64_t(sm_count) * 16;
  if (blocks < 1) blocks = 1;
  if (out_fp16)
    split_reduce_kernel<__half2><<<unsigned(blocks), 256, 0, s>>>(
        ws, static_cast<__half2*>(out), P, batch, splits, alpha, beta, chan_scale);
  else
    split_reduce_kernel<float2><<<unsigned(blocks), 256, 0, s>>>(
        ws, static_cast<float2*>(out), P, batch, splits, alpha, beta, chan_scale);
  return cudaGetLastError();
}

cudaError_t launch_herk_fp8(const CUtensorMap& tmZ, const HerkArgs& a, int grid, cudaStream_t s) {
  return a.out_fp16 ? launch_herk_t<__half, false>(tmZ, a, grid, s)
                    : launch_herk_t<float, false>(tmZ, a, grid, s);
}

cudaError_t launch_herk_fp8_fused(const CUtensorMap& tmQ, const HerkArgs& a, int grid,
                                  cudaStream_t s) {
  if (a.nseg != 1 || a.out_format != 0 || a.bulk_store || a.fp6 || a.s8)
    return cudaErrorInvalidValue;
  return a.out_fp16 ? launch_herk_t<__half, true>(tmQ, a, grid, s)
                    : launch_herk_t<float, true>(tmQ, a, grid, s);
}

}  // namespace ftdx
