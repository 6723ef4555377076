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
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "herk_fp8.cuh"

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
                                   int zpitch, int n, int batch, int split, float* qscale,
                                   float* out_scale, uint32_t* amax_bits, int sm_count,
                                   cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(amax_bits, 0, sizeof(uint32_t) * size_t(batch), s);
  if (e != cudaSuccess) return e;
  const int64_t per_chan = int64_t(n) * K;
  e = launch_channel_amax(a, per_chan, batch, amax_bits, sm_count, s);
  if (e != cudaSuccess) return e;
  scale_kernel<<<(batch + 127) / 128, 128, 0, s>>>(amax_bits, batch, qscale, out_scale);
  int rpb = 8192 / (Kp >> 3);
  if (rpb < 1) rpb = 1;
  const int64_t blocks = (rows + rpb - 1) / rpb;
  const int vec = (K % 2 == 0) && (reinterpret_cast<uintptr_t>(a) & 15) == 0;
  quantize_kernel<<<unsigned(blocks), 256, 0, s>>>(static_cast<const float2*>(a), z, rows, K, Kp,
                                                    zpitch, n, qscale, split, rpb, vec);
  return cudaGetLastError();
}

}  // namespace ftdx
