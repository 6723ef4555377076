// herk_fp4.cu -- NVFP4 correlator for float complex voltages.
//
// Quantisation (nvfp4_stats_kernel, nvfp4_order_kernel, nvfp4_quant_kernel): per input
// row a an FP32 scale g_a = amax_a / (6 * 448); per block of 16 values along
// K (8 complex samples, Re/Im interleaved) a UE4M3 block scale b >= amax_blk
// / (6 g_a) (rounded up, so no element saturates); elements E2M1(v / (g_a b)),
// round to nearest even.  Each input row a becomes two operand rows with the
// same block scales: x_a = (re, im)_t and y_a = (im, -re)_t, so that
//   x_j . x_i = Re R_ij and x_j . y_i = Im R_ij
// (the FP4 MMA has no negate bit; the sign lives in the y row).  The epilogue
// multiplies each product by g_i g_j; autocorrelations come from the exact
// FP64 row powers of the same pass.
//
// herk_fp4_tc_kernel: persistent tcgen05 kernel, tile = 128 column inputs j
// (MMA M, x rows) x 64 row inputs i (MMA N = 128: their x and y rows).  TMA
// brings per stage 128 B of K (256 E2M1 values) of A and B, and a bulk copy
// their four 512-byte scale atoms (written in that form by the quantiser);
// the MMA thread copies each atom into TMEM with tcgen05.cp (the layout
// tcgen05.mma kind::mxf4nvf4.block_scale reads: row m of a 128-row operand at
// lane m%32 of every lane quarter, column m/32, byte = the 16-element block
// within the 64-element k-step) and issues the MMAs (M=128, N=128, K=64)
// behind it in the same tcgen05 pipe; four epilogue warps store the packed
// triangle.
#include <cuda_fp4.h>
#include <cudaTypedefs.h>
#include <cuda_fp8.h>

#include <map>
#include <mutex>

#include "herk_fp8.cuh"
#include "sm100.cuh"

namespace ftdx {
using namespace dev;
namespace {

constexpr int k4J = 128;                      // j inputs per tile (A rows)
constexpr int k4I = 64;                       // i inputs per tile (B rows = 128)
constexpr int k4KB = 128;                     // operand bytes of K per stage (256 E2M1)
constexpr int k4Op = 128 * k4KB;              // 16 KB per operand per stage
constexpr int k4Sf = 128 * 16;                // 2 KB of scales per operand per stage
constexpr int k4StageBytes = 2 * k4Op + 2 * k4Sf;  // 36 KB (multiple of 1 KB)
constexpr int k4Stages = 5;
constexpr int k4AccCols = 128;                // (Re, Im) column pairs of 64 inputs
constexpr int k4SfCol0 = 2 * k4AccCols;       // TMEM columns of the scale-factor slots
constexpr int k4SfColsPerStage = 32;          // 4 k-steps x (4 SFA + 4 SFB) columns
constexpr int k4EpiWarps = 8;                 // two per TMEM lane quarter
constexpr int k4EpiGroups = k4EpiWarps / 4;   // warps per lane quarter (column chunks dealt round robin)
constexpr int k4Threads = 64 + 32 * k4EpiWarps;  // TMA, MMA, epilogue warps
constexpr size_t k4Smem = 1024 + size_t(k4Stages) * k4StageBytes + 256;

// E4M3 bits of a non-negative float, rounded up to the next representable
// value (the block scale must not let any element saturate).
__device__ __forceinline__ uint32_t ue4m3_ceil(float v) {
  if (!(v > 0.f)) return 0u;
  uint32_t c = uint32_t(__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3)) & 0x7Fu;
  const __half_raw h = __nv_cvt_fp8_to_halfraw(__nv_fp8_storage_t(c), __NV_E4M3);
  if (__half2float(__half(h)) < v && c < 0x7Eu) ++c;
  return c;
}
__device__ __forceinline__ float ue4m3_value(uint32_t c) {
  const __half_raw h = __nv_cvt_fp8_to_halfraw(__nv_fp8_storage_t(c), __NV_E4M3);
  return __half2float(__half(h));
}
__device__ __forceinline__ uint32_t fp4x2(float a, float b) {
  return uint32_t(__nv_cvt_float2_to_fp4x2(make_float2(a, b), __NV_E2M1, cudaRoundNearest));
}

// Block scales in the tcgen05 scale-factor atom: one 512-byte atom per 128
// operand rows and k-step (64 E2M1 values = 4 blocks); row m of the group at
// byte 16 (m % 32) + 4 (m / 32) + block.  A tcgen05.cp 32x128b.warpx4 of an
// atom gives the TMEM layout the block-scaled MMA reads (row m at lane
// m % 32 of every lane quarter, column m / 32, byte = block).  Groups are
// per channel and follow the kernel's tiles, so that one tile's rows are one
// group: A groups of 128 x rows; B groups of `gbrows` x/y rows (128 for the
// single-CTA kernel, 224 for the CTA pair), stored as `nsub` consecutive
// atoms per k-step (rows 0..127, 128..255 of the group).
struct SfGeom {
  int n;       // inputs per channel
  int gA;      // A groups per channel
  int gB;      // B groups per channel
  int nks;     // k-steps per row (both halves when split)
  int gbrows;  // operand rows per B group
  int nsub;    // atoms per B group and k-step: ceil(gbrows / 128)
};
__device__ __forceinline__ int64_t sf_atom_byte(int64_t group, int nks, int nsub, int ks, int m,
                                                int blk) {
  return ((group * nks + ks) * nsub + (m >> 7)) * 512 + (m & 31) * 16 + ((m >> 5) & 3) * 4 + blk;
}

// Values of a byte of two E2M1 codes (low nibble first).
__device__ __forceinline__ float2 fp4x2_value(uint32_t byte) {
  const __half2_raw h = __nv_cvt_fp4x2_to_halfraw2(__nv_fp4x2_storage_t(byte), __NV_E2M1);
  return __half22float2(__half2(h));
}

// E2M1 codes of x[0..15] * inv (round to nearest even, saturating at 6) into
// w (x = (re, im) byte order: element 2q in the low nibble of byte q) and
// the squared error sum of fl(d d), d = fma(-code, gb, x), in element order.
__device__ __forceinline__ float nvfp4_codes_err(const float (&x)[16], float inv, float gb,
                                                 uint32_t (&w)[2]) {
  w[0] = w[1] = 0u;
  float err = 0.f;
  const float2 inv2 = make_float2(inv, inv), gb2 = make_float2(gb, gb);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    // packed FP32 pairs: each component rounds as its scalar operation
    const float2 xq = make_float2(x[2 * q], x[2 * q + 1]);
    const float2 s = __fmul2_rn(xq, inv2);
    const uint32_t byte = fp4x2(s.x, s.y);
    w[q >> 2] |= byte << (8 * (q & 3));
    const float2 h = fp4x2_value(byte);
    const float2 d = __ffma2_rn(make_float2(-h.x, -h.y), gb2, xq);
    const float2 dd = __fmul2_rn(d, d);
    err = __fadd_rn(err, dd.x);
    err = __fadd_rn(err, dd.y);
  }
  return err;
}

// Quantise 16 values (8 complex samples, x[2q] = Re, x[2q+1] = Im) under the
// row's FP32 scale g into E2M1 codes of the x = (re, im) and y = (im, -re)
// operand rows.  The UE4M3 block scale is the better of two candidates by
// squared error: c0 = the smallest E4M3 value >= amax / (6 g) (no element
// saturates) and the next smaller code c0 - 1 when that is >= 1 (the largest
// element may saturate at 6, the rest land on a finer grid).  Every step is
// an explicitly rounded float32 operation (no contraction), so the choice is
// reproducible: gb = g b, inv = 1 / gb, codes = E2M1(x inv),
// err = sum of fl(d d) with d = fma(-code, gb, x); c0 - 1 wins only on a
// strictly smaller err.  Returns the chosen code; gb_out = g b of it.
__device__ __forceinline__ uint32_t nvfp4_quant16(const float (&x)[16], float g, uint32_t (&xw)[2],
                                                  uint32_t (&yw)[2], float& gb_out) {
  float amax = 0.f;
#pragma unroll
  for (int q = 0; q < 16; ++q) amax = fmaxf(amax, fabsf(x[q]));
  const uint32_t c0 = ue4m3_ceil(__fdiv_rn(amax, __fmul_rn(6.f, g)));
  const float gb0 = c0 ? __fmul_rn(g, ue4m3_value(c0)) : 0.f;
  const float err0 = nvfp4_codes_err(x, c0 ? __frcp_rn(gb0) : 0.f, gb0, xw);
  uint32_t best = c0;
  gb_out = gb0;
  if (c0 >= 2) {
    const float gb1 = __fmul_rn(g, ue4m3_value(c0 - 1));
    uint32_t w1[2];
    const float err1 = nvfp4_codes_err(x, __frcp_rn(gb1), gb1, w1);
    if (err1 < err0) {
      best = c0 - 1;
      gb_out = gb1;
      xw[0] = w1[0], xw[1] = w1[1];
    }
  }
  // y = (im, -re): swap the nibbles of every byte and flip the sign bit of
  // the new high nibble (-0 for a zero code: the same value in the MMA)
#pragma unroll
  for (int h = 0; h < 2; ++h)
    yw[h] = (((xw[h] & 0x0F0F0F0Fu) ^ 0x08080808u) << 4) | ((xw[h] >> 4) & 0x0F0F0F0Fu);
  return best;
}

// Where one input row's quantiser output goes: its x and y operand rows
// (hi half of pitch bytes, lo half after it) and its three scale bytes of
// k-step 0, block 0 (sf_atom_byte: the x row in sfa, the x and y rows in
// sfb); k-step ks, block blk is at + ks * 512 + blk in sfa and at
// + ks * sbk + blk in sfb, the lo k-steps ksh after the hi ones.
struct Fp4RowOut {
  uint8_t* zx;
  uint8_t* zy;
  uint8_t* sa;
  uint8_t* sbx;
  uint8_t* sby;
  int sbk;    // sfb bytes per k-step: nsub atoms of 512
  int ksh;    // k-steps per half
  int pitch;  // bytes per half of an operand row
};
__device__ __forceinline__ Fp4RowOut fp4_row_out(int64_t r, int c, int w, uint8_t* z,
                                                 uint8_t* sfa, uint8_t* sfb, int pitch,
                                                 const SfGeom& sg) {
  Fp4RowOut o;
  o.zx = z + (2 * r) * int64_t(2 * pitch);
  o.zy = o.zx + 2 * pitch;
  const int64_t ga = int64_t(c) * sg.gA + (w >> 7);
  const int64_t gbk = int64_t(c) * sg.gB + (2 * w) / sg.gbrows;
  const int ob = (2 * w) % sg.gbrows;  // x row in the group; y row next (gbrows is even)
  o.sa = sfa + sf_atom_byte(ga, sg.nks, 1, 0, w & 127, 0);
  o.sbx = sfb + sf_atom_byte(gbk, sg.nks, sg.nsub, 0, ob, 0);
  o.sby = sfb + sf_atom_byte(gbk, sg.nks, sg.nsub, 0, ob + 1, 0);
  o.sbk = sg.nsub * 512;
  o.ksh = pitch / 32;
  o.pitch = pitch;
  return o;
}

// One 16-value block b of an input row: the hi codes and, when `lo`, the
// residual r = fma(-code, g b, x) quantised again with its own block scale
// (same g), written where `o` says.
__device__ __forceinline__ void nvfp4_block(const float (&x)[16], float g, int b,
                                            const Fp4RowOut& o, bool lo) {
  uint32_t xw[2], yw[2];
  float gb = 0.f;
  const uint32_t bc = nvfp4_quant16(x, g, xw, yw, gb);
  *reinterpret_cast<uint2*>(o.zx + 8 * b) = make_uint2(xw[0], xw[1]);
  *reinterpret_cast<uint2*>(o.zy + 8 * b) = make_uint2(yw[0], yw[1]);
  const int ks = b >> 2, blk = b & 3;
  o.sa[ks * 512 + blk] = uint8_t(bc);
  o.sbx[ks * o.sbk + blk] = uint8_t(bc);
  o.sby[ks * o.sbk + blk] = uint8_t(bc);
  if (lo) {  // the residual fma(-code, g b, x) quantised with its own block scale
    float res[16];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float2 h = fp4x2_value((xw[q >> 2] >> (8 * (q & 3))) & 0xFFu);
      const float2 r2 = __ffma2_rn(make_float2(-h.x, -h.y), make_float2(gb, gb),
                                   make_float2(x[2 * q], x[2 * q + 1]));
      res[2 * q] = r2.x;
      res[2 * q + 1] = r2.y;
    }
    uint32_t xl[2], yl[2];
    float gb2 = 0.f;
    const uint32_t bc2 = nvfp4_quant16(res, g, xl, yl, gb2);
    *reinterpret_cast<uint2*>(o.zx + o.pitch + 8 * b) = make_uint2(xl[0], xl[1]);
    *reinterpret_cast<uint2*>(o.zy + o.pitch + 8 * b) = make_uint2(yl[0], yl[1]);
    const int kl = o.ksh + ks;
    o.sa[kl * 512 + blk] = uint8_t(bc2);
    o.sbx[kl * o.sbk + blk] = uint8_t(bc2);
    o.sby[kl * o.sbk + blk] = uint8_t(bc2);
  }
}

// Pass 1, one warp per input row: max |Re|, |Im| (the row's FP32 scale
// g_r = amax_r / (6 * 448), 1 for an empty row; NaN counts as 0) and the
// autocorrelation sum_t |v_t|^2 (FP64, fixed order, so deterministic).  With
// `rfi`, a second read of the row (from L2) flags the time samples with
// |v_t|^2 > 25 x the row's mean power in the channel's bitmap.
constexpr double kRfiThreshold = 25.0;
__global__ void __launch_bounds__(256) nvfp4_stats_kernel(
    const float2* __restrict__ a, float* __restrict__ power, float* __restrict__ rscale,
    uint32_t* __restrict__ flags, int64_t rows, int K, int n, int fwords, int rfi) {
  const int lane = threadIdx.x & 31;
  // rows of an even K at a 16-byte aligned base: two samples per load
  const bool vec = (K & 1) == 0 && (reinterpret_cast<uintptr_t>(a) & 15) == 0;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += (int64_t(gridDim.x) * blockDim.x) >> 5) {
    const float2* p = a + r * K;
    double acc = 0.0, emax = 0.0;  // sum and largest of |v_t|^2 (each exact in FP64 before the sum)
    float m = 0.f;
    auto take = [&](float x, float y) {
      const double e = double(x) * x + double(y) * y;
      acc += e;
      emax = fmax(emax, e);
      m = fmaxf(m, fmaxf(fabsf(x), fabsf(y)));
    };
    if (vec) {
      const float4* p4 = reinterpret_cast<const float4*>(p);
      const int k2 = K >> 1;
      for (int t0 = lane; t0 < k2; t0 += 128) {  // four 16-byte loads in flight per lane
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          v[u] = (t0 + 32 * u < k2) ? __ldg(p4 + t0 + 32 * u) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          take(v[u].x, v[u].y);
          take(v[u].z, v[u].w);
        }
      }
    } else {
      for (int t0 = lane; t0 < K; t0 += 128) {  // four loads in flight per lane
        float2 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          v[u] = (t0 + 32 * u < K) ? __ldg(p + t0 + 32 * u) : make_float2(0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 4; ++u) take(v[u].x, v[u].y);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      acc += __shfl_xor_sync(0xffffffffu, acc, o);
      emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
      m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if (lane == 0) {
      power[r] = float(acc);
      rscale[r] = (m > 0.f && m < 3.0e38f) ? m / (6.f * 448.f) : 1.f;
    }
    const double thr = kRfiThreshold * acc / double(K);
    // a row none of whose samples exceeds the threshold (every Gaussian row)
    // sets no flag: the second read is skipped
    if (rfi && acc > 0.0 && emax > thr) {
      uint32_t* f = flags + (r / n) * fwords;
      for (int t0 = lane; t0 < K; t0 += 128) {  // four loads in flight per lane
        float2 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          v[u] = (t0 + 32 * u < K) ? __ldg(p + t0 + 32 * u) : make_float2(0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int t = t0 + 32 * u;
          if (t < K && double(v[u].x) * v[u].x + double(v[u].y) * v[u].y > thr)
            atomicOr(f + (t >> 5), 1u << (t & 31));
        }
      }
    }
  }
}

// Pass 2, one block per channel: the channel's time order and lo extent.
// Plain mode with F flagged samples: position (number of unflagged samples
// before t) for an unflagged t, K - F + (number of flagged samples before t)
// for a flagged one -- a correlation is invariant under a common permutation
// of time, and the flagged samples (impulsive RFI, which E2M1 with one
// mantissa bit renders worst) land together in the last stages, which alone
// carry a lo residual.  src[p] = the source sample of position p (-1:
// padding); nflag[c] = F; chans[c].pad = number of trailing k-blocks (of
// 128 samples) with a lo residual (all of them in split mode).
__global__ void __launch_bounds__(1024) nvfp4_order_kernel(const uint32_t* __restrict__ flags,
                                                           int32_t* __restrict__ src,
                                                           int32_t* __restrict__ nflag,
                                                           ChanDesc* __restrict__ chans, int K,
                                                           int kp, int fwords, int split) {
  __shared__ int s_cnt[32];
  __shared__ int s_total;
  const int c = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const uint32_t* f = flags + int64_t(c) * fwords;
  int cnt = 0;
  if (!split)
    for (int x = threadIdx.x; x < fwords; x += blockDim.x) cnt += __popc(f[x]);
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0) s_cnt[warp] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int x = 0; x < nwarps; ++x) tot += s_cnt[x];
    s_total = tot;
  }
  __syncthreads();
  const int F = s_total;
  const int kblocks = kp / 128;
  if (threadIdx.x == 0) {
    nflag[c] = F;
    chans[c].pad = split ? kblocks : (F == 0 ? 0 : kblocks - (K - F) / 128);
  }
  int32_t* sc = src + int64_t(c) * kp;
  for (int p = K + threadIdx.x; p < kp; p += blockDim.x) sc[p] = -1;
  if (F == 0) {
    for (int t = threadIdx.x; t < K; t += blockDim.x) sc[t] = t;
    return;
  }
  int base = 0;  // flagged samples before this chunk
  for (int t0 = 0; t0 < K; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    const bool fl = t < K && ((f[t >> 5] >> (t & 31)) & 1u);
    const uint32_t bal = __ballot_sync(0xffffffffu, fl);
    __syncthreads();  // s_cnt of the previous chunk consumed
    if (lane == 0) s_cnt[warp] = __popc(bal);
    __syncthreads();
    int before = base + __popc(bal & ((1u << lane) - 1u));
    int chunk = 0;
    for (int x = 0; x < nwarps; ++x) {
      if (x < warp) before += s_cnt[x];
      chunk += s_cnt[x];
    }
    if (t < K) sc[fl ? (K - F + before) : (t - before)] = t;
    base += chunk;
  }
}

// Pass 3, one warp per input row: the E2M1 operands and UE4M3 scale atoms in
// the channel's time order (lane l: blocks l, l + 32, ...), with the lo
// residual in the blocks of the trailing chans[c].pad k-blocks.
__global__ void __launch_bounds__(256, 4) nvfp4_quant_kernel(
    const float2* __restrict__ a, const int32_t* __restrict__ src,
    const int32_t* __restrict__ nflag, const ChanDesc* __restrict__ chans,
    const float* __restrict__ rscale, uint8_t* __restrict__ z, uint8_t* __restrict__ sfa,
    uint8_t* __restrict__ sfb, int64_t rows, int K, int kp, int pitch, SfGeom sg) {
  const int lane = threadIdx.x & 31;
  const int blocks_per_row = pitch / 8;  // 8 bytes of E2M1 per block
  const bool vec = (K & 1) == 0 && (reinterpret_cast<uintptr_t>(a) & 15) == 0;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += (int64_t(gridDim.x) * blockDim.x) >> 5) {
    const float2* p = a + r * K;
    const float g = __ldg(rscale + r);
    const int c = int(r / sg.n), w = int(r - int64_t(c) * sg.n);
    const bool permuted = __ldg(nflag + c) > 0;
    const int lo_from = (kp / 128 - chans[c].pad) * 16;  // first block with a residual
    const int32_t* sc = src + int64_t(c) * kp;
    const Fp4RowOut o = fp4_row_out(r, c, w, z, sfa, sfb, pitch, sg);
    for (int b = lane; b < blocks_per_row; b += 32) {
      const int t0 = 8 * b;
      float x[16];
      if (!permuted && vec && t0 + 8 <= K) {
        const float4* p4 = reinterpret_cast<const float4*>(p + t0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 v = __ldg(p4 + q);
          x[4 * q] = v.x, x[4 * q + 1] = v.y, x[4 * q + 2] = v.z, x[4 * q + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int t = permuted ? (t0 + q < kp ? __ldg(sc + t0 + q) : -1) : (t0 + q < K ? t0 + q : -1);
          const float2 v = t >= 0 ? __ldg(p + t) : make_float2(0.f, 0.f);
          x[2 * q] = v.x, x[2 * q + 1] = v.y;
        }
      }
      nvfp4_block(x, g, b, o, b >= lo_from);
    }
  }
}

// Block-scaled instruction descriptor: E2M1 x E2M1, UE4M3 scales, FP32
// accumulate, K-major A and B, K = 64.
constexpr uint32_t idesc_nvf4(uint32_t M, uint32_t N) {
  return (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

struct Fp4Args {
  const TileDesc* tiles;
  const ChanDesc* chans;
  int num_tiles;
  void* out;
  float alpha, beta;
  const float* row_scale;  // g_r per input row (the products carry g_i g_j)
  uint32_t* status;
  const float* row_power;  // exact sum_t |v_t|^2 per input row (the autocorrelations)
  const uint8_t* sfa;      // scale atoms of the x rows (A)
  const uint8_t* sfb;      // scale atoms of the x/y rows (B)
  int gA, gB, nks;         // SfGeom: groups per channel, k-steps per row
  // k-blocks from a row's hi half to its lo half (the lo residual of the
  // channel's trailing ChanDesc::pad k-blocks; see fp4_segment)
  int lo_off;
};

// k-block kb of a channel's K loop -> (A k-block, B k-block): first the
// kbl hi x hi k-blocks, then `lo` k-blocks of hi x lo (B's lo half, L k-blocks
// into the row) and `lo` of lo x hi, both over the channel's last `lo`
// k-blocks (ChanDesc::pad, written by nvfp4_order_kernel; lo x lo is left out).
__device__ __forceinline__ void fp4_segment(int kb, int kbl, int lo, int L, int& ka, int& kbb) {
  if (kb < kbl) {
    ka = kbb = kb;
    return;
  }
  const int m = kb - kbl, base = kbl - lo;
  if (m < lo) {
    ka = base + m;
    kbb = L + base + m;
  } else {
    ka = L + base + (m - lo);
    kbb = base + (m - lo);
  }
}

// Epilogue of one 32-column accumulator chunk: rows i0..i0+15 (columns 2m,
// 2m+1 = Re, Im of row i0+m) of lane j's column.  Element (i, j <= i < n)
// = r * alpha g_i g_j (+ beta * old), the diagonal the exact row power;
// sc_j = alpha g_j, gl = g_(i0 + lane % 16) (prefetched; the 16 row scales
// reach every lane by warp shuffles); chunks wholly below the diagonal and
// inside n store unmasked.  Row i0+m of the packed triangle starts
// m i0 + m(m+1)/2 after row i0.
__device__ __forceinline__ void fp4_store_chunk(float2* __restrict__ outc, const uint32_t (&r)[32],
                                                int i0, int j, int jw, int n, float sc_j, float gl,
                                                const float* __restrict__ pw, float alpha,
                                                float beta) {
  const bool interior = (i0 + 15 < n) && (jw + 31 < i0);
  float2* p0 = outc + int64_t(i0) * (i0 + 1) / 2 + j;
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const float s = sc_j * __shfl_sync(0xffffffffu, gl, m);  // alpha g_i g_j
    const int i = i0 + m;
    if (interior || (i < n && j <= i)) {
      float2* p = p0 + (int64_t(m) * i0 + m * (m + 1) / 2);
      float vr, vi;
      if (!interior && i == j) {
        // autocorrelations come from the FP64 power pass: their NVFP4 estimate
        // would carry the quantisation-noise power as a bias
        vr = __ldg(pw + i) * alpha;
        vi = 0.f;
      } else {
        vr = __uint_as_float(r[2 * m]) * s;
        vi = __uint_as_float(r[2 * m + 1]) * s;
      }
      if (beta != 0.f) {
        const float2 o = *p;
        vr += beta * o.x;
        vi += beta * o.y;
      }
      __stcs(p, make_float2(vr, vi));
    }
  }
}

// Row scales one epilogue warp needs for one tile: alpha g_j of its lane's
// column and g_i of row i0 + lane % 16 for each of its accumulator chunks.
template <int kChunksPerWarp>
struct Fp4TileScales {
  float sc_j;
  float gl[kChunksPerWarp];
};

// The epilogue warps' tile loop of both NVFP4 kernels.  A warp drains TMEM
// lane quarter q (32 columns j) of each accumulator, chunks grp, grp +
// kEpiGroups, ... of 32 columns (16 rows i).  The global loads a tile needs
// run ahead of its accumulator: tile and channel descriptors two tiles ahead,
// row scales one tile ahead, so that no tile's stores wait on a load (the
// MMAs of a tile take about as long as one descriptor -> channel -> scale
// chain of dependent loads).
//   jt: inputs j per tile (TileDesc::tj unit); jo: this CTA's first j in it;
//   it: inputs i per tile; kCols: accumulator columns (2 per input i).
template <int kCols>
__device__ __forceinline__ void fp4_epilogue(const Fp4Args& args, uint32_t tmem_base, int first,
                                             int stride, int jt, int jo, int it, int q, int grp,
                                             int lane, uint32_t tfull0, uint32_t tempty0,
                                             bool cluster_release, volatile int* abort_flag) {
  constexpr int kChunks = kCols / 32;
  constexpr int kPer = (kChunks + k4EpiGroups - 1) / k4EpiGroups;
  using Scales = Fp4TileScales<kPer>;
  const int nt = args.num_tiles;
  float2* out = static_cast<float2*>(args.out);
  auto load_scales = [&](const TileDesc& td, const ChanDesc& cd) {
    Scales sv;
    const int j = int(td.tj) * jt + jo + q * 32 + lane;
    sv.sc_j = args.alpha * (j < cd.n ? __ldg(args.row_scale + cd.row0 + j) : 0.f);
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int c = grp + k * k4EpiGroups;
      const int il = int(td.ti) * it + 16 * c + (lane & 15);
      sv.gl[k] = (c < kChunks && il < cd.n) ? __ldg(args.row_scale + cd.row0 + il) : 0.f;
    }
    return sv;
  };
  int t = first;
  if (t >= nt) return;
  TileDesc td0 = args.tiles[t];
  ChanDesc cd0 = args.chans[td0.ch];
  TileDesc td1 = t + stride < nt ? args.tiles[t + stride] : td0;
  ChanDesc cd1 = args.chans[td1.ch];
  Scales s0 = load_scales(td0, cd0);
  int acc = 0;
  uint32_t acc_phase = 0;
  for (; t < nt; t += stride) {
    const TileDesc td2 = t + 2 * stride < nt ? args.tiles[t + 2 * stride] : td1;
    const Scales s1 = load_scales(td1, cd1);
    const uint32_t tfull = tfull0 + 8u * uint32_t(acc);
    const bool ok = __all_sync(0xffffffffu, mbar_wait(tfull, acc_phase, abort_flag));
    if (!ok) {
      if (lane == 0) atomicOr(args.status, kStatusTimeoutEpilogue);
      break;
    }
    tc_fence_after();
    const int n = cd0.n;
    const int jw = int(td0.tj) * jt + jo + q * 32;
    const int j = jw + lane;
    const int ib = int(td0.ti) * it;
    float2* outc = out + cd0.out0;
    const uint32_t tb = tmem_base + (uint32_t(q * 32) << 16) + uint32_t(acc * kCols);
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int c = grp + k * k4EpiGroups;
      if (c >= kChunks) break;
      const int i0 = ib + 16 * c;
      if (i0 + 15 < jw || i0 >= n) continue;  // warp-uniform: nothing to store
      uint32_t r[32];
      __syncwarp();
      tmem_ld_32x32b_x32(tb + 32u * c, r);
      tmem_wait_ld();
      fp4_store_chunk(outc, r, i0, j, jw, n, s0.sc_j, s0.gl[k], args.row_power + cd0.row0,
                      args.alpha, args.beta);
    }
    tc_fence_before();
    __syncwarp();
    if (lane == 0) {
      const uint32_t te = tempty0 + 8u * uint32_t(acc);
      if (cluster_release)
        mbar_arrive_cluster_relaxed(map_shared(te, 0));
      else
        mbar_arrive(te);
    }
    if (++acc == 2) {
      acc = 0;
      acc_phase ^= 1u;
    }
    const ChanDesc cd2 = args.chans[td2.ch];
    td0 = td1;
    cd0 = cd1;
    s0 = s1;
    td1 = td2;
    cd1 = cd2;
  }
}

__global__ void __launch_bounds__(k4Threads, 1)
    herk_fp4_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                       const Fp4Args args) {
  extern __shared__ uint8_t smem_dyn[];
  uint8_t* smem = smem_dyn + ((1024u - (smem_u32(smem_dyn) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + k4Stages * k4StageBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * k4Stages + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const uint32_t smem0 = smem_u32(smem);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (k4Stages + s); };
  auto tfull_bar = [&](int b) { return bar0 + 8u * (3 * k4Stages + b); };
  auto tempty_bar = [&](int b) { return bar0 + 8u * (3 * k4Stages + 2 + b); };
  const uint32_t done_bar = bar0 + 8u * (3 * k4Stages + 4);
  auto a_addr = [&](int s) { return smem0 + uint32_t(s * k4StageBytes); };
  auto b_addr = [&](int s) { return smem0 + uint32_t(s * k4StageBytes + k4Op); };
  auto sfa_addr = [&](int s) { return smem0 + uint32_t(s * k4StageBytes + 2 * k4Op); };
  auto sfb_addr = [&](int s) { return smem0 + uint32_t(s * k4StageBytes + 2 * k4Op + k4Sf); };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < k4Stages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull_bar(b), 1);
      mbar_init(tempty_bar(b), k4EpiWarps);
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
  }
  if (warp == 1) {
    tmem_alloc(smem_u32(tmem_slot), 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------ TMA producer
    if (lane == 0) {
      int stage = 0, issued = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
        const TileDesc td = args.tiles[t];
        const ChanDesc cd = args.chans[td.ch];
        const int32_t rowA = int32_t(cd.row0 + int64_t(td.tj) * k4J);        // x-row view
        const int32_t rowB = int32_t(2 * (cd.row0 + int64_t(td.ti) * k4I));  // all rows
        const uint8_t* sfA = args.sfa + (int64_t(td.ch) * args.gA + td.tj) * args.nks * 512;
        const uint8_t* sfB = args.sfb + (int64_t(td.ch) * args.gB + td.ti) * args.nks * 512;
        for (int kb = 0; kb < cd.kblocks + 2 * cd.pad; ++kb) {
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutProducer);
            ok = false;
            break;
          }
          int ka, kbb;
          fp4_segment(kb, cd.kblocks, cd.pad, args.lo_off, ka, kbb);
          mbar_arrive_expect_tx(full_bar(stage), k4StageBytes);
          tma_load_2d(a_addr(stage), &tmA, ka * k4KB, rowA, full_bar(stage));
          tma_load_2d(b_addr(stage), &tmB, kbb * k4KB, rowB, full_bar(stage));
          bulk_load(sfa_addr(stage), sfA + int64_t(ka) * 4 * 512, k4Sf, full_bar(stage));
          bulk_load(sfb_addr(stage), sfB + int64_t(kbb) * 4 * 512, k4Sf, full_bar(stage));
          ++issued;
          if (++stage == k4Stages) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) {
        int s = stage;
        uint32_t ph = phase;
        for (int q = 0; q < k4Stages && q < issued; ++q) {
          if (--s < 0) {
            s = k4Stages - 1;
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
      constexpr uint32_t idesc = idesc_nvf4(128, 128);
      int stage = 0, acc = 0;
      uint32_t phase = 0, acc_phase = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
        const ChanDesc cd = args.chans[args.tiles[t].ch];
        if (!mbar_wait(tempty_bar(acc), acc_phase ^ 1u, abort_flag)) {
          atomicOr(args.status, kStatusTimeoutMma);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + uint32_t(acc * k4AccCols);
        for (int kb = 0; kb < cd.kblocks + 2 * cd.pad; ++kb) {
          if (!mbar_wait(full_bar(stage), phase, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutMma);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sf0 = tmem_base + uint32_t(k4SfCol0 + stage * k4SfColsPerStage);
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            tmem_cp_32x128b_warpx4(sf0 + 4 * s, sdesc_none_kmajor(sfa_addr(stage) + 512 * s, 128));
            tmem_cp_32x128b_warpx4(sf0 + 16 + 4 * s,
                                   sdesc_none_kmajor(sfb_addr(stage) + 512 * s, 128));
          }
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            mma_nvf4(d, sdesc_sw128_kmajor(a_addr(stage) + 32 * s),
                     sdesc_sw128_kmajor(b_addr(stage) + 32 * s), idesc, sf0 + 4 * s,
                     sf0 + 16 + 4 * s, (kb | s) != 0);
          }
          mma_commit(empty_bar(stage));
          if (++stage == k4Stages) {
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
      mma_commit(done_bar);
      volatile int never = 0;
      if (!mbar_wait(done_bar, 0, &never)) atomicOr(args.status, kStatusTimeoutOther);
    }
  } else {
    // ------------------------------------------------ epilogue (warps 2..)
    // warp w drains lane quarter w % 4, column chunks c = (w - 2) / 4 mod groups
    fp4_epilogue<k4AccCols>(args, tmem_base, blockIdx.x, gridDim.x, k4J, 0, k4I, warp & 3,
                            (warp - 2) >> 2, lane, tfull_bar(0), tempty_bar(0), false,
                            abort_flag);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem_base, 512);
  }
}

// ---------------------------------------------------------------- CTA pair
// herk_fp4_pair_kernel: the same product on a CTA pair (cluster of 2), as the
// FP8 pair kernel.  Tile = 256 column inputs j (MMA M = 256: 128 x rows per
// CTA) x 112 row inputs i (MMA N = 224: their x and y rows, 112 per CTA), so
// each CTA's shared memory feeds twice the MMA work per operand byte of the
// single-CTA kernel.  Every load of both CTAs completes on the leader's full
// barrier; the leader's MMA thread copies each stage's scale atoms into both
// CTAs' TMEM (tcgen05.cp.cta_group::2: each CTA from its own shared memory;
// SFA = its own 128 rows, SFB = all 224 rows, loaded by both) and issues the
// MMAs behind them in the same pipe, so one TMEM scale slot per stage
// suffices: 2 x 224 accumulator columns + 16 SFA + 32 SFB columns of 512.
constexpr int k4pJ = 256;                     // j inputs per pair tile
constexpr int k4pI = 112;                     // i inputs per pair tile
constexpr int k4pN = 2 * k4pI;                // MMA N: x/y rows of the i inputs
constexpr int k4pA = 128 * k4KB;              // 16 KB: this CTA's 128 x rows
constexpr int k4pB = k4pI * k4KB;             // 14 KB: this CTA's 112 x/y rows
constexpr int k4pSfa = 4 * 512;               // 4 k-steps x one atom
constexpr int k4pSfb = 4 * 2 * 512;           // 4 k-steps x two atoms (224 rows)
constexpr int k4pStageBytes = k4pA + k4pB + k4pSfa + k4pSfb;  // 36 KB (multiple of 1 KB)
constexpr int k4pStages = 6;
constexpr int k4pAccCols = k4pN;              // one accumulator: 224 columns
constexpr int k4pSfaCol = 2 * k4pAccCols;     // 448: 4 k-steps x 4 columns
constexpr int k4pSfbCol = k4pSfaCol + 16;     // 464: 4 k-steps x 8 columns (..495)
constexpr int k4pThreads = 64 + 32 * k4EpiWarps;  // TMA, MMA, epilogue warps
constexpr size_t k4pSmem = 1024 + size_t(k4pStages) * k4pStageBytes + 256;
static_assert(k4pSfbCol + 32 <= 512, "TMEM columns");

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(k4pThreads, 1)
    herk_fp4_pair_kernel(const __grid_constant__ CUtensorMap tmA,
                         const __grid_constant__ CUtensorMap tmB,
                         const __grid_constant__ CUtensorMap tmSa,
                         const __grid_constant__ CUtensorMap tmSb, const Fp4Args args) {
  extern __shared__ uint8_t smem_dyn[];
  uint8_t* smem = smem_dyn + ((1024u - (smem_u32(smem_dyn) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + k4pStages * k4pStageBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * k4pStages + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const uint32_t smem0 = smem_u32(smem);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (k4pStages + s); };
  auto tfull_bar = [&](int b) { return bar0 + 8u * (2 * k4pStages + b); };
  auto tempty_bar = [&](int b) { return bar0 + 8u * (2 * k4pStages + 2 + b); };
  const uint32_t done_bar = bar0 + 8u * (2 * k4pStages + 4);
  auto a_addr = [&](int s) { return smem0 + uint32_t(s * k4pStageBytes); };
  auto b_addr = [&](int s) { return smem0 + uint32_t(s * k4pStageBytes + k4pA); };
  auto sfa_addr = [&](int s) { return smem0 + uint32_t(s * k4pStageBytes + k4pA + k4pB); };
  auto sfb_addr = [&](int s) {
    return smem0 + uint32_t(s * k4pStageBytes + k4pA + k4pB + k4pSfa);
  };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const int pair = int(blockIdx.x >> 1), npairs = int(gridDim.x >> 1);
  if (threadIdx.x == 0) {
    for (int s = 0; s < k4pStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull_bar(b), 1);
      mbar_init(tempty_bar(b), 2 * k4EpiWarps);  // the epilogue warps of both CTAs
    }
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
    tma_prefetch_desc(&tmSa);
    tma_prefetch_desc(&tmSb);
  }
  if (warp == 1) {
    tmem_alloc_pair(smem_u32(tmem_slot), 512);
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
      for (int t = pair; t < args.num_tiles; t += npairs) {
        const TileDesc td = args.tiles[t];
        const ChanDesc cd = args.chans[td.ch];
        const int32_t rowA = int32_t(cd.row0 + int64_t(td.tj) * k4pJ + 128 * rank);  // x rows
        const int32_t rowB = int32_t(2 * cd.row0 + int64_t(td.ti) * k4pN + k4pI * rank);
        const int64_t ga = int64_t(td.ch) * args.gA + 2 * int64_t(td.tj) + rank;
        const int64_t gb = int64_t(td.ch) * args.gB + td.ti;
        bool ok = true;
        for (int kb = 0; kb < cd.kblocks + 2 * cd.pad; ++kb) {
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutProducer);
            ok = false;
            break;
          }
          int ka, kbb;
          fp4_segment(kb, cd.kblocks, cd.pad, args.lo_off, ka, kbb);
          if (leader) mbar_arrive_expect_tx(full_bar(stage), 2 * k4pStageBytes);
          const uint32_t fb = map_shared(full_bar(stage), 0);
          tma_load_2d_pair(a_addr(stage), &tmA, ka * k4KB, rowA, fb);
          tma_load_2d_pair(b_addr(stage), &tmB, kbb * k4KB, rowB, fb);
          // scale atoms as rows of 256 bytes: SFA (ga, 4 ka ..): 8 rows, SFB: 16
          tma_load_2d_pair(sfa_addr(stage), &tmSa, 0, int32_t((ga * args.nks + 4 * ka) * 2), fb);
          tma_load_2d_pair(sfb_addr(stage), &tmSb, 0, int32_t((gb * args.nks + 4 * kbb) * 4), fb);
          if (++stage == k4pStages) {
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
      constexpr uint32_t idesc = idesc_nvf4(256, k4pN);
      const uint32_t sfa_t = tmem_base + uint32_t(k4pSfaCol);
      const uint32_t sfb_t = tmem_base + uint32_t(k4pSfbCol);
      int stage = 0, acc = 0;
      uint32_t phase = 0, acc_phase = 0;
      bool ok = true;
      for (int t = pair; t < args.num_tiles && ok; t += npairs) {
        const ChanDesc cd = args.chans[args.tiles[t].ch];
        if (!mbar_wait(tempty_bar(acc), acc_phase ^ 1u, abort_flag)) {
          atomicOr(args.status, kStatusTimeoutMma);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + uint32_t(acc * k4pAccCols);
        for (int kb = 0; kb < cd.kblocks + 2 * cd.pad; ++kb) {
          if (!mbar_wait(full_bar(stage), phase, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutMma);
            ok = false;
            break;
          }
          tc_fence_after();
          // the previous stage's MMAs read these columns: the copies queue
          // behind them in the tcgen05 pipe
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            tmem_cp_32x128b_warpx4_pair(sfa_t + 4 * s,
                                        sdesc_none_kmajor(sfa_addr(stage) + 512 * s, 128));
            tmem_cp_32x128b_warpx4_pair(sfb_t + 8 * s,
                                        sdesc_none_kmajor(sfb_addr(stage) + 1024 * s, 128));
            tmem_cp_32x128b_warpx4_pair(sfb_t + 8 * s + 4,
                                        sdesc_none_kmajor(sfb_addr(stage) + 1024 * s + 512, 128));
          }
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            mma_nvf4_pair(d, sdesc_sw128_kmajor(a_addr(stage) + 32 * s),
                          sdesc_sw128_kmajor(b_addr(stage) + 32 * s), idesc, sfa_t + 4 * s,
                          sfb_t + 8 * s, (kb | s) != 0);
          }
          mma_commit_pair_both(empty_bar(stage));
          if (++stage == k4pStages) {
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
    // ------------------------------------------------ epilogue (warps 2.., both CTAs)
    // warp w drains lane quarter w % 4, column chunks c = (w - 2) / 4 mod groups;
    // both CTAs release an accumulator on the leader's barrier
    fp4_epilogue<k4pAccCols>(args, tmem_base, pair, npairs, k4pJ, 128 * int(rank), k4pI,
                             warp & 3, (warp - 2) >> 2, lane, tfull_bar(0), tempty_bar(0), true,
                             abort_flag);
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // neither CTA leaves while the other may still signal it
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, 512);
  }
}

}  // namespace

namespace {
// Workspace carve-up of one NVFP4 call (every part 1 KB aligned): E2M1
// operand rows (2 per input, each a hi half and a lo half of `pitch` bytes),
// the scale atoms of the A and B views, the row powers and row scales, the
// channels' RFI bitmaps, flagged counts and time orders.
struct Fp4Ws {
  int64_t pitch, rpitch;   // E2M1 bytes per operand row: one half, whole row
  int64_t kp;              // samples per row, padded to the 128-sample stage
  int fwords;              // 32-bit words of one channel's RFI bitmap
  SfGeom sg;
  int64_t z_bytes, sfa_bytes, sfb_bytes, pw_bytes, flag_bytes, nflag_bytes, src_bytes, total;
};
Fp4Ws fp4_ws(int n, int batch, int K, int pair) {
  Fp4Ws w;
  const int64_t rows = int64_t(n) * batch;
  w.pitch = (2 * int64_t(K) + 255) / 256 * 128;
  w.rpitch = 2 * w.pitch;
  w.kp = w.pitch;  // samples per padded row: two E2M1 values a byte, two a sample
  w.fwords = int((K + 31) / 32);
  const int nks = int(w.rpitch / 32);
  if (pair)  // A: both 128-row halves of every 256-input tile; B: 224-row groups
    w.sg = SfGeom{n, 2 * ((n + k4pJ - 1) / k4pJ), (2 * n + k4pN - 1) / k4pN, nks, k4pN, 2};
  else
    w.sg = SfGeom{n, (n + 127) / 128, (2 * n + 127) / 128, nks, 128, 1};
  auto up = [](int64_t b) { return (b + 1023) / 1024 * 1024; };
  w.z_bytes = up(2 * rows * w.rpitch);
  w.sfa_bytes = up(int64_t(batch) * w.sg.gA * w.sg.nks * 512);
  w.sfb_bytes = up(int64_t(batch) * w.sg.gB * w.sg.nks * w.sg.nsub * 512);
  w.pw_bytes = up(4 * rows);
  w.flag_bytes = up(int64_t(batch) * w.fwords * 4);
  w.nflag_bytes = up(int64_t(batch) * 4);
  w.src_bytes = up(int64_t(batch) * w.kp * 4);
  w.total = w.z_bytes + w.sfa_bytes + w.sfb_bytes + 2 * w.pw_bytes + w.flag_bytes +
            w.nflag_bytes + w.src_bytes;
  return w;
}
}  // namespace

// Workspace: E2M1 operand rows (2 per input; twice as long when split), the
// scale atoms of the A and B views, the row powers and the row scales.
size_t nvfp4_workspace_bytes(int n, int batch, int K, int split, int pair) {
  (void)split;  // one layout for both modes: every row has room for its lo half
  return size_t(fp4_ws(n, batch, K, pair).total);
}

// Pairs of the NVFP4 pair kernel that can be resident at once on the current
// device (0: none), queried once per device.
int nvfp4_pair_limit() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  static std::mutex mu;
  static std::map<int, int> limits;
  std::lock_guard<std::mutex> lock(mu);
  auto it = limits.find(dev);
  if (it != limits.end()) return it->second;
  int limit = 0;
  if (ensure_smem_limit(reinterpret_cast<const void*>(herk_fp4_pair_kernel), k4pSmem) ==
      cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2, 1, 1);
    cfg.blockDim = dim3(k4pThreads, 1, 1);
    cfg.dynamicSmemBytes = k4pSmem;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, herk_fp4_pair_kernel, &cfg) == cudaSuccess) limit = n;
  }
  cudaGetLastError();
  limits[dev] = limit;
  return limit;
}

// Tile list of the pair kernel for one channel of n inputs: tj over 256
// column inputs, ti over 112 row inputs, tiles holding some j <= i.
void nvfp4_pair_tiles(int n, int ch, std::vector<TileDesc>& out) {
  const int ni = (n + k4pI - 1) / k4pI, nj = (n + k4pJ - 1) / k4pJ;
  for (int ti = 0; ti < ni; ++ti)
    for (int tj = 0; tj < nj && tj * k4pJ <= ti * k4pI + k4pI - 1; ++tj)
      out.push_back(TileDesc{ch, uint16_t(ti), uint16_t(tj)});
}

int nvfp4_kblocks(int K) { return int((2 * int64_t(K) + 255) / 256); }

cudaError_t launch_nvfp4(const void* A, int64_t rows, int K, int n, int batch, uint8_t* ws,
                         const TileDesc* tiles, const ChanDesc* chans, int num_tiles, void* C,
                         float alpha, float beta, uint32_t* status, int sm_count, void* encode_fn,
                         cudaStream_t s, int split, int pair, int phases) {
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(encode_fn);
  if (!encode) return cudaErrorInvalidValue;
  if (pair && nvfp4_pair_limit() < 1) return cudaErrorInvalidConfiguration;
  const Fp4Ws w = fp4_ws(n, batch, K, pair);
  const int64_t pitch = w.pitch, rpitch = w.rpitch;  // one half (hi or lo), whole row
  uint8_t* z = ws;
  uint8_t* sfa = ws + w.z_bytes;
  uint8_t* sfb = sfa + w.sfa_bytes;
  float* power = reinterpret_cast<float*>(sfb + w.sfb_bytes);
  float* rscale = reinterpret_cast<float*>(sfb + w.sfb_bytes + w.pw_bytes);
  uint32_t* flags = reinterpret_cast<uint32_t*>(sfb + w.sfb_bytes + 2 * w.pw_bytes);
  int32_t* nflag = reinterpret_cast<int32_t*>(reinterpret_cast<uint8_t*>(flags) + w.flag_bytes);
  int32_t* src = reinterpret_cast<int32_t*>(reinterpret_cast<uint8_t*>(nflag) + w.nflag_bytes);
  // rows of a partial group get no scales from the quantiser: zero them
  // (their products land only in outputs the epilogue skips)
  cudaError_t e;
  if (phases & 1) {  // the quantiser passes
    if (n % (pair ? k4pJ : 128) != 0 || (2 * n) % w.sg.gbrows != 0) {
      e = cudaMemsetAsync(sfa, 0, size_t(w.sfa_bytes + w.sfb_bytes), s);
      if (e != cudaSuccess) return e;
    }
    const int rfi = split ? 0 : 1;
    if (rfi) {
      e = cudaMemsetAsync(flags, 0, size_t(w.flag_bytes), s);
      if (e != cudaSuccess) return e;
    }
    int64_t blocks = (rows + 7) / 8;  // one warp per row
    if (blocks > int64_t(sm_count) * 16) blocks = int64_t(sm_count) * 16;
    // row scales, row powers and (plain mode) the channels' RFI bitmaps
    nvfp4_stats_kernel<<<unsigned(blocks), 256, 0, s>>>(static_cast<const float2*>(A), power,
                                                        rscale, flags, rows, K, n, w.fwords, rfi);
    // time order and lo extent of every channel (written into the plan's table)
    nvfp4_order_kernel<<<unsigned(batch), 1024, 0, s>>>(flags, src, nflag,
                                                        const_cast<ChanDesc*>(chans), K,
                                                        int(w.kp), w.fwords, split);
    // E2M1 operands and UE4M3 scale atoms
    nvfp4_quant_kernel<<<unsigned(blocks), 256, 0, s>>>(static_cast<const float2*>(A), src, nflag,
                                                        chans, rscale, z, sfa, sfb, rows, K,
                                                        int(w.kp), int(pitch), w.sg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (!(phases & 2)) return cudaSuccess;

  CUtensorMap tmA, tmB, tmSa, tmSb;
  const cuuint32_t estr[2] = {1, 1};
  auto enc2 = [&](CUtensorMap* m, void* base, int64_t inner, int64_t nrows, int64_t stride,
                  uint32_t box0, CUtensorMapSwizzle sw, uint32_t box1 = 128) {
    const cuuint64_t dims[2] = {cuuint64_t(inner), cuuint64_t(nrows)};
    const cuuint64_t str[1] = {cuuint64_t(stride)};
    const cuuint32_t box[2] = {box0, box1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, str, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  };
  if (enc2(&tmA, z, rpitch, rows, 2 * rpitch, k4KB, CU_TENSOR_MAP_SWIZZLE_128B) != CUDA_SUCCESS ||
      enc2(&tmB, z, rpitch, 2 * rows, rpitch, k4KB, CU_TENSOR_MAP_SWIZZLE_128B,
           pair ? k4pI : 128) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  if (pair &&  // scale atoms as rows of 256 bytes: 4 atoms (SFA) / 8 atoms (SFB) per stage
      (enc2(&tmSa, sfa, 256, w.sfa_bytes / 256, 256, 256, CU_TENSOR_MAP_SWIZZLE_NONE, 8) !=
           CUDA_SUCCESS ||
       enc2(&tmSb, sfb, 256, w.sfb_bytes / 256, 256, 256, CU_TENSOR_MAP_SWIZZLE_NONE, 16) !=
           CUDA_SUCCESS))
    return cudaErrorInvalidValue;
  Fp4Args args{tiles, chans, num_tiles, C, alpha, beta, rscale, status, power,
               sfa, sfb, w.sg.gA, w.sg.gB, w.sg.nks};
  args.lo_off = int(pitch / k4KB);  // hi . lo + lo . hi over each channel's lo k-blocks
  if (pair) {
    const int limit = nvfp4_pair_limit();
    const int pairs = num_tiles < limit ? num_tiles : limit;
    herk_fp4_pair_kernel<<<2 * pairs, k4pThreads, k4pSmem, s>>>(tmA, tmB, tmSa, tmSb, args);
    return cudaGetLastError();
  }
  e = ensure_smem_limit(reinterpret_cast<const void*>(herk_fp4_tc_kernel), k4Smem);
  if (e != cudaSuccess) return e;
  const int grid = num_tiles < sm_count ? num_tiles : sm_count;
  herk_fp4_tc_kernel<<<grid, k4Threads, k4Smem, s>>>(tmA, tmB, args);
  return cudaGetLastError();
}

}  // namespace ftdx
