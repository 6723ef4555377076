// precision.cu -- promotion of float complex voltages to the FP8 operand
// planes with a per-channel scale, plain or split into hi + lo parts.
//
//   amax pass   : per channel, the largest |Re| or |Im| (atomicMax on the
//                 bit patterns of non-negative floats, which order like ints)
//   scale pass  : s_c = 448 / amax_c (448 = largest finite E4M3); the
//                 correlator multiplies channel c's result by 1 / s_c^2
//   quantise    : hi = E4M3(s_c x) (round to nearest even, saturating) into
//                 columns [0, Kp) of the planes; in split mode also
//                 lo = E4M3(s_c x - hi) into columns [Kp, 2 Kp).  With the
//                 correlator's K segments (hi,hi) + (hi,lo) + (lo,hi) this
//                 carries about 7 significant bits per sample instead of 4.
//
// In the plain mode the three passes run as one cooperative persistent
// kernel (scale_quantize_kernel) when the device can hold its grid: each
// block takes the same share of every channel, finds the amax of its share
// of channel c while it quantises its share of channel c - 1, which it read
// one channel earlier and which is still in L2, so HBM sees the input once.
// The split mode, and a grid that cannot be co-resident, use three kernels
// (amax, scale, quantise) that read it twice.
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <mutex>

#include "herk_fp8.cuh"
#include "sm100.cuh"

namespace ftdx {
namespace {

// Per channel c (blockIdx.y): the largest |Re| or |Im|.  Each thread reads
// two samples (16 bytes) per load, four loads in flight; `vec` (uniform)
// says the channel starts 16-byte aligned and per_chan is even.
__global__ void __launch_bounds__(256) amax_kernel(const float2* __restrict__ a, int64_t per_chan,
                                                   uint32_t* __restrict__ amax_bits, int vec) {
  const int c = blockIdx.y;
  const float2* p = a + int64_t(c) * per_chan;
  float m = 0.f;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (vec) {
    const float4* p4 = reinterpret_cast<const float4*>(p);
    const int64_t n4 = per_chan >> 1;
    int64_t i = t0;
    for (; i + 3 * stride < n4; i += 4 * stride) {
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = __ldg(p4 + i + u * stride);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        m = fmaxf(m, fmaxf(fmaxf(fabsf(v[u].x), fabsf(v[u].y)), fmaxf(fabsf(v[u].z), fabsf(v[u].w))));
    }
    for (; i < n4; i += stride) {
      const float4 v = __ldg(p4 + i);
      m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
    }
  } else {
    for (int64_t i = t0; i < per_chan; i += stride) {
      const float2 v = __ldg(p + i);
      m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
    }
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < int(blockDim.x >> 5); ++w) m = fmaxf(m, wm[w]);
    if (!(m == m)) m = 0.f;  // NaN input: treat as empty
    atomicMax(amax_bits + c, __float_as_uint(m));
  }
}

__global__ void scale_kernel(const uint32_t* __restrict__ amax_bits, int batch,
                             float* __restrict__ qscale, float* __restrict__ out_scale) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= batch) return;
  const float m = __uint_as_float(amax_bits[c]);
  const float s = (m > 0.f && m < 3.0e38f) ? 448.f / m : 1.f;
  qscale[c] = s;
  out_scale[c] = 1.f / (s * s);
}

__device__ __forceinline__ uint32_t e4m3x2(float a, float b) {
  return uint32_t(__nv_cvt_float2_to_fp8x2(make_float2(a, b), __NV_SATFINITE, __NV_E4M3));
}
__device__ __forceinline__ float e4m3_to_float(uint32_t byte) {
  const __half_raw hr = __nv_cvt_fp8_to_halfraw(__nv_fp8_storage_t(byte), __NV_E4M3);
  return __half2float(__half(hr));
}

// One thread quantises 8 samples of one row.  With `vec` (uniform: K even
// and the input 16-byte aligned) a row's 8 samples are read as four 16-byte
// loads; otherwise, and past K, one sample at a time.
__global__ void __launch_bounds__(256) quantize_kernel(const float2* __restrict__ a,
                                                       uint8_t* __restrict__ z, int64_t rows,
                                                       int K, int Kp, int zpitch, int n,
                                                       const float* __restrict__ qscale, int split,
                                                       int rows_per_block, int vec) {
  const int chunks = Kp >> 3;
  const int64_t r0 = int64_t(blockIdx.x) * rows_per_block;
  const int64_t nrows64 = rows - r0 < rows_per_block ? rows - r0 : rows_per_block;
  const int nloc = int(nrows64) * chunks;
  const int64_t plane = rows * int64_t(zpitch);
  // the block's rows belong to at most a few channels: 32-bit channel index
  const int c0 = int(r0 / n), rin0 = int(r0 - int64_t(c0) * n);
  for (int l = threadIdx.x; l < nloc; l += blockDim.x) {
    const int rl = l / chunks;
    const int t0 = (l - rl * chunks) << 3;
    const int64_t r = r0 + rl;
    const float s = qscale[c0 + (rin0 + rl) / n];
    float xr[8], xi[8];
    const float2* src = a + r * K + t0;
    if (vec && t0 + 8 <= K) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(src) + q);
        xr[2 * q] = v.x * s;
        xi[2 * q] = v.y * s;
        xr[2 * q + 1] = v.z * s;
        xi[2 * q + 1] = v.w * s;
      }
    } else {
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const float2 v = (t0 + b < K) ? __ldg(src + b) : make_float2(0.f, 0.f);
        xr[b] = v.x * s;
        xi[b] = v.y * s;
      }
    }
    uint32_t hr[2], hi_[2], lr[2], li[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const float* pr = xr + 4 * q;
      const float* pi = xi + 4 * q;
      hr[q] = e4m3x2(pr[0], pr[1]) | (e4m3x2(pr[2], pr[3]) << 16);
      hi_[q] = e4m3x2(pi[0], pi[1]) | (e4m3x2(pi[2], pi[3]) << 16);
      if (split) {
        float dr[4], di[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          dr[b] = pr[b] - e4m3_to_float((hr[q] >> (8 * b)) & 0xFFu);
          di[b] = pi[b] - e4m3_to_float((hi_[q] >> (8 * b)) & 0xFFu);
        }
        lr[q] = e4m3x2(dr[0], dr[1]) | (e4m3x2(dr[2], dr[3]) << 16);
        li[q] = e4m3x2(di[0], di[1]) | (e4m3x2(di[2], di[3]) << 16);
      }
    }
    uint8_t* dst = z + r * zpitch + t0;
    *reinterpret_cast<uint2*>(dst) = make_uint2(hr[0], hr[1]);
    *reinterpret_cast<uint2*>(dst + plane) = make_uint2(hi_[0], hi_[1]);
    if (split) {
      *reinterpret_cast<uint2*>(dst + Kp) = make_uint2(lr[0], lr[1]);
      *reinterpret_cast<uint2*>(dst + plane + Kp) = make_uint2(li[0], li[1]);
    }
  }
}

// L2 policy that makes lines the first to be evicted (for data read for
// the last time).  The loads that use it allocate in L1 at evict-first
// priority: a thread's four 16-byte loads of a unit fall into sectors that
// neighbouring lanes share, and the second load of each sector then hits L1
// (85.1 against 87.7 us at 8 channels with no L1 allocation).
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ float4 ldg_last_use(const float4* p, uint64_t pol) {
  float4 v;
  asm volatile("ld.global.nc.L1::evict_first.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p), "l"(pol));
  return v;
}

// The 8 samples t0 .. t0 + 7 of one row (src = the row + t0) as Re and Im
// arrays; samples at or past K read as 0.  pol != 0: an L2 policy for the
// 16-byte loads (the samples' last use).
__device__ __forceinline__ void load_unit(const float2* __restrict__ src, int t0, int K, bool vec,
                                          float (&xr)[8], float (&xi)[8], uint64_t pol = 0) {
  if (vec && t0 + 8 <= K) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4* p4 = reinterpret_cast<const float4*>(src) + q;
      const float4 v = pol ? ldg_last_use(p4, pol) : __ldg(p4);
      xr[2 * q] = v.x, xi[2 * q] = v.y, xr[2 * q + 1] = v.z, xi[2 * q + 1] = v.w;
    }
  } else {
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const float2 v = (t0 + b < K) ? __ldg(src + b) : make_float2(0.f, 0.f);
      xr[b] = v.x, xi[b] = v.y;
    }
  }
}

// (row, unit column) of unit u0 + threadIdx.x of a channel of `chunks` units
// per row, advanced by blockDim.x units per next() without a division.
struct UnitWalk {
  int row, col, drow, dcol, chunks;
  __device__ __forceinline__ UnitWalk(int64_t u0, int chunks_) : chunks(chunks_) {
    const int u = int(u0) + int(threadIdx.x);
    row = u / chunks;
    col = u - row * chunks;
    drow = int(blockDim.x) / chunks;
    dcol = int(blockDim.x) - drow * chunks;
  }
  __device__ __forceinline__ void next() {
    row += drow;
    col += dcol;
    if (col >= chunks) col -= chunks, ++row;
  }
  __device__ __forceinline__ int t0() const { return col << 3; }
  // offsets of the unit's first sample in a channel's input ([n][K]) and
  // planes (pitch zpitch)
  __device__ __forceinline__ int64_t offset(int K) const { return int64_t(row) * K + (col << 3); }
  __device__ __forceinline__ int64_t zoffset(int zpitch) const {
    return int64_t(row) * zpitch + (col << 3);
  }
};

// Number of units of the block range starting at u0 (per_blk units, cut at
// the channel's end; 0 past it).
__device__ __forceinline__ int u1_len(int64_t u0, int64_t per_blk, int64_t units) {
  const int64_t u1 = u0 + per_blk < units ? u0 + per_blk : units;
  return u1 > u0 ? int(u1 - u0) : 0;
}

// Thread 0 of a block of scale_quantize_kernel: wait until every block has
// counted its amax of channel cq into its arrival word (acquire; bounded by
// FTDX_WAIT_NS, after which the status word gets kStatusTimeoutOther and the
// block's later waits are skipped), then the channel's scale s = 448 / amax
// as scale_kernel (block 0 also stores qscale and out_scale).
__device__ __forceinline__ float wait_channel_scale(int cq, float* __restrict__ qscale,
                                                    float* __restrict__ out_scale,
                                                    uint32_t* amax_bits, uint32_t* arrive_word,
                                                    uint32_t* status, bool& aborted) {
  if (!aborted && !dev::flag_wait_limit(arrive_word, gridDim.x, FTDX_WAIT_NS)) {
    atomicOr(status, dev::kStatusTimeoutOther);
    aborted = true;
  }
  uint32_t mb;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(mb) : "l"(amax_bits + cq) : "memory");
  const float mx = __uint_as_float(mb);
  const float sc = (mx > 0.f && mx < 3.0e38f) ? 448.f / mx : 1.f;
  if (blockIdx.x == 0) {
    qscale[cq] = sc;
    out_scale[cq] = 1.f / (sc * sc);
  }
  return sc;
}

// Quantise one unit (8 samples, Re xr / Im xi) with scale sc into the planes
// at dst (plane 1 at + plane, plane 2 = -plane 0 at + 2 plane when neg), with
// quantize_kernel's arithmetic; streaming stores (the planes are not read
// again by this kernel).
__device__ __forceinline__ void quantise_unit(float (&xr)[8], float (&xi)[8], float sc,
                                              uint8_t* __restrict__ dst, int64_t plane, int neg) {
#pragma unroll
  for (int b = 0; b < 8; ++b) xr[b] *= sc, xi[b] *= sc;
  uint32_t hr[2], hi_[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    hr[q] = e4m3x2(xr[4 * q], xr[4 * q + 1]) | (e4m3x2(xr[4 * q + 2], xr[4 * q + 3]) << 16);
    hi_[q] = e4m3x2(xi[4 * q], xi[4 * q + 1]) | (e4m3x2(xi[4 * q + 2], xi[4 * q + 3]) << 16);
  }
  constexpr uint32_t kS = 0x80808080u;
  __stcs(reinterpret_cast<uint2*>(dst), make_uint2(hr[0], hr[1]));
  __stcs(reinterpret_cast<uint2*>(dst + plane), make_uint2(hi_[0], hi_[1]));
  if (neg) __stcs(reinterpret_cast<uint2*>(dst + 2 * plane), make_uint2(hr[0] ^ kS, hr[1] ^ kS));
}

// Channel amax, scale and quantisation in one cooperative launch (every
// block resident: the blocks wait on one another).  A channel is n rows x
// Kp / 8 units of 8 samples; block b owns the same contiguous unit range of
// every channel, and thread t the units L[k] = t + k blockDim.x of it
// (k < cnt).  With p = ceil(cnt / 2), step c (0 .. batch) is:
//   1. amax over L[0 .. p) of channel c, two units per round trip;
//   2. thread 0 waits for channel c - 1's amax (wait_channel_scale);
//   3. amax over L[p .. cnt) of channel c, each beside the quantisation of
//      L[k] of channel c - 1 (k = 0 ..), both loads in flight together;
//   4. the block's amax of channel c into amax_bits[c] (atomicMax on the
//      bits, as amax_kernel), and the block counted into channel c's
//      arrival word (release; one 128-byte line per channel, so the blocks
//      polling channel c - 1 do not contend with these atomics);
//   5. the rest of channel c - 1's units quantised, two per round trip.
// Two block barriers per step (after 2 and inside 4); the shared scale and
// warp maxima alternate between two slots by step parity, so a step needs
// no closing barrier.  A unit is re-read about one channel of reads (n K
// samples) after its first read, so the re-read hits L2 while a channel is
// well below the L2's size.  neg: also write plane 2 = plane 0 with every
// sign flipped.  Per-element arithmetic is that of the three-kernel path,
// so both give the same bits.
__global__ void __launch_bounds__(256, 4) scale_quantize_kernel(
    const float2* __restrict__ a, uint8_t* __restrict__ z, int K, int Kp, int zpitch, int n,
    int batch, int neg, float* __restrict__ qscale, float* __restrict__ out_scale,
    uint32_t* amax_bits, uint32_t* arrive, uint32_t* status, int vec) {
  const int chunks = Kp >> 3;
  const int64_t units = int64_t(n) * chunks;
  const int64_t per_blk = (units + gridDim.x - 1) / gridDim.x;
  const int64_t u0 = int64_t(blockIdx.x) * per_blk;
  const int len = u1_len(u0, per_blk, units);
  const int t = int(threadIdx.x), bd = int(blockDim.x);
  const int cnt = t < len ? (len - t + bd - 1) / bd : 0;  // this thread's units
  const int p = (cnt + 1) / 2;
  const int64_t plane = int64_t(n) * batch * zpitch;
  const int64_t chan_in = int64_t(n) * K, chan_z = int64_t(n) * zpitch;
  const uint64_t pol = l2_evict_first_policy();  // channel c - 1's samples: read for the last time
  __shared__ float wm[2][8];
  __shared__ float s_scale[2];
  bool aborted = false;  // thread 0's
  for (int c = 0; c <= batch; ++c) {
    const bool amax_step = c < batch, quant_step = c >= 1;
    const int par = c & 1;
    const float2* cur = a + int64_t(amax_step ? c : 0) * chan_in;        // channel c (amax)
    const float2* prev = a + int64_t(quant_step ? c - 1 : 0) * chan_in;  // channel c - 1
    uint8_t* zprev = z + int64_t(quant_step ? c - 1 : 0) * chan_z;
    float m = 0.f;
    float xr[8], xi[8], yr[8], yi[8];
    UnitWalk wa(u0, chunks), wb(u0, chunks);
    auto amax_of = [&](const float (&r)[8], const float (&im)[8]) {
#pragma unroll
      for (int b = 0; b < 8; ++b) m = fmaxf(m, fmaxf(fabsf(r[b]), fabsf(im[b])));
    };
    int ka = 0, kb = 0;  // next L index of the amax / quantisation walks
    float sc = 1.f;
    if (amax_step) {  // 1
      const int kend = quant_step ? p : cnt;  // the first step has nothing to wait for
      for (; ka + 1 < kend; ka += 2) {
        UnitWalk w2 = wa;
        w2.next();
        load_unit(cur + wa.offset(K), wa.t0(), K, vec, xr, xi);
        load_unit(cur + w2.offset(K), w2.t0(), K, vec, yr, yi);
        amax_of(xr, xi);
        amax_of(yr, yi);
        w2.next();
        wa = w2;
      }
      if (ka < kend) {
        load_unit(cur + wa.offset(K), wa.t0(), K, vec, xr, xi);
        amax_of(xr, xi);
        wa.next();
        ++ka;
      }
    }
    if (quant_step) {
      if (t == 0)  // 2
        s_scale[par] = wait_channel_scale(c - 1, qscale, out_scale, amax_bits,
                                          arrive + int64_t(c - 1) * 32, status, aborted);
      __syncthreads();
      sc = s_scale[par];
      if (amax_step) {  // 3
        for (; ka < cnt; ++ka, ++kb) {
          load_unit(cur + wa.offset(K), wa.t0(), K, vec, xr, xi);
          load_unit(prev + wb.offset(K), wb.t0(), K, vec, yr, yi, pol);
          amax_of(xr, xi);
          quantise_unit(yr, yi, sc, zprev + wb.zoffset(zpitch), plane, neg);
          wa.next();
          wb.next();
        }
      }
    }
    if (amax_step) {  // 4
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      if ((t & 31) == 0) wm[par][t >> 5] = m;
      __syncthreads();
      if (t == 0) {
        for (int x = 1; x < (bd >> 5); ++x) m = fmaxf(m, wm[par][x]);
        if (!(m == m)) m = 0.f;
        atomicMax(amax_bits + c, __float_as_uint(m));
        __threadfence();
        atomicAdd(arrive + int64_t(c) * 32, 1u);
      }
    }
    if (quant_step) {  // 5
      for (; kb + 1 < cnt; kb += 2) {
        UnitWalk w2 = wb;
        w2.next();
        load_unit(prev + wb.offset(K), wb.t0(), K, vec, xr, xi, pol);
        load_unit(prev + w2.offset(K), w2.t0(), K, vec, yr, yi, pol);
        quantise_unit(xr, xi, sc, zprev + wb.zoffset(zpitch), plane, neg);
        quantise_unit(yr, yi, sc, zprev + w2.zoffset(zpitch), plane, neg);
        w2.next();
        wb = w2;
      }
      if (kb < cnt) {
        load_unit(prev + wb.offset(K), wb.t0(), K, vec, xr, xi, pol);
        quantise_unit(xr, xi, sc, zprev + wb.zoffset(zpitch), plane, neg);
      }
    }
  }
}

// Blocks of scale_quantize_kernel per SM that can be resident (0: unknown).
int scale_quantize_blocks_per_sm() {
  static std::once_flag once;
  static int nb = 0;
  std::call_once(once, [] {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, scale_quantize_kernel, 256, 0) !=
        cudaSuccess) {
      nb = 0;
      cudaGetLastError();
    }
  });
  return nb;
}

}  // namespace

cudaError_t launch_channel_amax(const void* a, int64_t per_chan, int batch, uint32_t* amax_bits,
                                int sm_count, cudaStream_t s) {
  // about 8 blocks of 256 threads per SM over all channels, each thread with
  // at least 4 x 16-byte loads
  int bx = int((per_chan + 256 * 8 - 1) / (256 * 8));
  const int cap = (sm_count * 8 + batch - 1) / batch;
  if (bx > cap) bx = cap;
  if (bx < 1) bx = 1;
  const int vec = (per_chan % 2 == 0) && (reinterpret_cast<uintptr_t>(a) & 15) == 0;
  amax_kernel<<<dim3(unsigned(bx), unsigned(batch)), 256, 0, s>>>(static_cast<const float2*>(a),
                                                                   per_chan, amax_bits, vec);
  return cudaGetLastError();
}

cudaError_t launch_float_to_planes(const void* a, uint8_t* z, int64_t rows, int K, int Kp,
                                   int zpitch, int n, int batch, int split, int neg,
                                   float* qscale, float* out_scale, uint32_t* amax_bits,
                                   uint32_t* arrive, uint32_t* status, int sm_count,
                                   cudaStream_t s) {
  // the arrival words (32 per channel) directly followed by amax_bits: one
  // memset zeroes both
  const bool adjacent = amax_bits == arrive + int64_t(batch) * 32;
  cudaError_t e = adjacent ? cudaMemsetAsync(arrive, 0, sizeof(uint32_t) * size_t(batch) * 33, s)
                           : cudaMemsetAsync(amax_bits, 0, sizeof(uint32_t) * size_t(batch), s);
  if (e != cudaSuccess) return e;
  const int vec = (K % 2 == 0) && (reinterpret_cast<uintptr_t>(a) & 15) == 0;
  const int64_t units = int64_t(n) * (Kp >> 3);
  // the split mode (hi and lo columns) measured faster on the three-kernel
  // path: 0.91 against 1.02 ms at 4096 x 64 x 1024
  const int per_sm = split ? 0 : scale_quantize_blocks_per_sm();
  if (per_sm > 0 && adjacent && (reinterpret_cast<uintptr_t>(arrive) & 127) == 0 &&
      units < (int64_t(1) << 30)) {
    // at least 256 units (one per thread) per block, at most every resident block
    int64_t grid = (units + 255) / 256;
    if (grid > int64_t(per_sm) * sm_count) grid = int64_t(per_sm) * sm_count;
    if (grid < 1) grid = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, scale_quantize_kernel, static_cast<const float2*>(a), z, K, Kp,
                           zpitch, n, batch, neg, qscale, out_scale, amax_bits, arrive, status,
                           vec);
    if (e == cudaSuccess) return e;
    cudaGetLastError();  // not launchable as one cooperative grid: the three-kernel path
  }
  const int64_t per_chan = int64_t(n) * K;
  e = launch_channel_amax(a, per_chan, batch, amax_bits, sm_count, s);
  if (e != cudaSuccess) return e;
  scale_kernel<<<(batch + 127) / 128, 128, 0, s>>>(amax_bits, batch, qscale, out_scale);
  int rpb = 8192 / (Kp >> 3);
  if (rpb < 1) rpb = 1;
  const int64_t blocks = (rows + rpb - 1) / rpb;
  quantize_kernel<<<unsigned(blocks), 256, 0, s>>>(static_cast<const float2*>(a), z, rows, K, Kp,
                                                    zpitch, n, qscale, split, rpb, vec);
  e = cudaGetLastError();
  if (e == cudaSuccess && neg) e = launch_negate_plane(z, rows * zpitch, sm_count, s);
  return e;
}

}  // namespace ftdx
