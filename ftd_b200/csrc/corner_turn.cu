// corner_turn.cu -- operand promotion straight from raw packet-ordered QC
// voltages: the corner turn into per-(channel, pol, time_inner) antenna rows
// and the QC -> FP8 E4M3 conversion in one pass, writing the correlator's
// Re / Im (/ -Re) planes Z[planes][rows][Kp].
//
// Reference layouts (paths within cpviolator/ftd):
//   [t][ant][chan][pol], t = k*n_ti + ti: cpu_herk_ftd,
//     tests/visibility_pipeline_test.cpp:55-96;
//   [chan][pol][ant][t], t = ti*K + k: qc_pol_gather_transpose_kernel,
//     lib/bench_pipeline.cu:306-331.
// Output row of source sample (ant, chan, pol, ti, k):
//   row = b*n_ant + ant, b = (chan*n_pol + pol)*n_ti + ti,  column k;
//   pol_sum: b = chan*n_ti + ti, column pol*K + k (one HERK over n_pol*K).
// Columns [n_seg*K, Kp) of every row are zero (n_seg = n_pol with pol_sum,
// else 1).
#include <cuda_runtime.h>

#include "herk_fp8.cuh"
#include "qc_codec.cuh"

namespace ftdx {
namespace {

constexpr int kTK = 128;         // time samples per tile
constexpr int kTS = 128;         // source bytes (ant, chan, pol) per tile
constexpr int kTPitch = kTK + 4; // transposed tile row pitch (bytes)

__device__ __forceinline__ void put32(uint8_t* dst, const uint32_t (&w)[8], int nbytes) {
  // nbytes valid bytes of the 32 at dst (any alignment)
  if (nbytes == 32 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
    reinterpret_cast<uint4*>(dst)[0] = make_uint4(w[0], w[1], w[2], w[3]);
    reinterpret_cast<uint4*>(dst)[1] = make_uint4(w[4], w[5], w[6], w[7]);
  } else if (nbytes == 32 && (reinterpret_cast<uintptr_t>(dst) & 3) == 0) {
#pragma unroll
    for (int x = 0; x < 8; ++x) reinterpret_cast<uint32_t*>(dst)[x] = w[x];
  } else {
#pragma unroll
    for (int b = 0; b < 32; ++b)  // unrolled: w stays in registers
      if (b < nbytes) dst[b] = uint8_t(w[b >> 2] >> (8 * (b & 3)));
  }
}

// [t][ant][chan][pol] source.  Block (x, y, z): source bytes [128 x, +128) of
// a time slice (S = n_ant*n_chan*n_pol bytes each), samples k in [128 y, +128),
// time_inner z.  The 128 x 128 byte tile is read with coalesced 4-byte loads
// along the slice, transposed 4 x 4 in registers into shared memory as
// [source byte][k], then every (source byte, 32 samples) run is converted and
// written as 32 contiguous bytes per plane (four threads: one 128-byte line).
// Eight blocks per SM (32 registers, a few bytes spilled) beat six (40
// registers, no spill): the kernel is latency- and issue-bound.
__global__ void __launch_bounds__(256, 8) ftd_tacp_to_planes_kernel(const uint8_t* __restrict__ raw,
                                                                 uint8_t* __restrict__ z,
                                                                 FtdGeom g) {
  __shared__ __align__(16) uint8_t tileT[kTS * kTPitch];
  const int64_t S = int64_t(g.n_ant) * g.n_chan * g.n_pol;
  const int64_t s0 = int64_t(blockIdx.x) * kTS;
  const int k0 = blockIdx.y * kTK;
  const int ti = blockIdx.z;
  const int t = threadIdx.x;
  const bool wide = (S & 3) == 0 && (reinterpret_cast<uintptr_t>(raw) & 3) == 0;
  // phase 1: kTK / 4 k-groups x 32 s-groups of 4 x 4 bytes, kTK / 32 per thread
#pragma unroll
  for (int rep = 0; rep < kTK / 32; ++rep) {
    const int blk = t + 256 * rep;
    const int sg = blk & 31, kg = blk >> 5;  // lanes of a warp: consecutive source words
    uint32_t w[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int k = k0 + 4 * kg + r;
      const int64_t s = s0 + 4 * sg;
      uint32_t v = 0;
      if (k < g.K) {
        const uint8_t* src = raw + (g.t_stride ? int64_t(k) * g.t_stride + ti * g.z_stride
                                               : (int64_t(k) * g.n_ti + ti) * S) + s;
        if (wide && s + 4 <= S) {
          v = __ldg(reinterpret_cast<const uint32_t*>(src));
        } else {
          for (int b = 0; b < 4; ++b)
            if (s + b < S) v |= uint32_t(__ldg(src + b)) << (8 * b);
        }
      }
      w[r] = v;  // byte b = source s + b at sample k0 + 4 kg + r
    }
    // transpose: out[b] byte r = w[r] byte b
    const uint32_t lo01 = __byte_perm(w[0], w[1], 0x5140), hi01 = __byte_perm(w[0], w[1], 0x7362);
    const uint32_t lo23 = __byte_perm(w[2], w[3], 0x5140), hi23 = __byte_perm(w[2], w[3], 0x7362);
    const uint32_t o0 = __byte_perm(lo01, lo23, 0x5410), o1 = __byte_perm(lo01, lo23, 0x7632);
    const uint32_t o2 = __byte_perm(hi01, hi23, 0x5410), o3 = __byte_perm(hi01, hi23, 0x7632);
    uint8_t* d = tileT + (4 * sg) * kTPitch + 4 * kg;
    *reinterpret_cast<uint32_t*>(d) = o0;
    *reinterpret_cast<uint32_t*>(d + kTPitch) = o1;
    *reinterpret_cast<uint32_t*>(d + 2 * kTPitch) = o2;
    *reinterpret_cast<uint32_t*>(d + 3 * kTPitch) = o3;
  }
  __syncthreads();
  // phase 2: task -> (source byte sl, samples [32 h, +32)), kTK / 64 per thread
#pragma unroll 1
  for (int task = t; task < kTS * (kTK / 32); task += 256) {
    const int sl = task / (kTK / 32), h = task % (kTK / 32);
    const int64_t s = s0 + sl;
    if (s >= S) break;
    // 32-bit divisions (S < 2^31, checked at launch): the 64-bit ones are
    // emulated in dozens of instructions each
    const uint32_t s32 = uint32_t(s);
    const int pol = int(s32 % uint32_t(g.n_pol));
    const uint32_t ac = s32 / uint32_t(g.n_pol);
    const int chan = int(ac % uint32_t(g.n_chan));
    const int ant = int(ac / uint32_t(g.n_chan));
    int64_t row;
    int col0, kend;
    if (g.pol_sum) {
      row = (int64_t(chan) * g.n_ti + ti) * g.n_ant + ant;
      col0 = pol * g.K;
      kend = (pol == g.n_pol - 1) ? g.Kp - (g.n_pol - 1) * g.K : g.K;  // last pol owns the padding
    } else {
      row = ((int64_t(chan) * g.n_pol + pol) * g.n_ti + ti) * g.n_ant + ant;
      col0 = 0;
      kend = g.Kp;
    }
    const int kb = k0 + 32 * h;
    if (kb >= kend) continue;
    const int nbytes = kend - kb < 32 ? kend - kb : 32;
    uint32_t q[8];
    const uint8_t* src = tileT + sl * kTPitch + 32 * h;
#pragma unroll
    for (int x = 0; x < 8; ++x) q[x] = *reinterpret_cast<const uint32_t*>(src + 4 * x);
    uint32_t re[8], im[8];
    if (g.twos) {
#pragma unroll
      for (int x = 0; x < 8; ++x) tc4_to_e4m3(q[x], re[x], im[x]);
    } else {
#pragma unroll
      for (int x = 0; x < 8; ++x) qc4_to_e4m3(q[x], re[x], im[x]);
    }
    const int64_t plane = g.rows * int64_t(g.Kp);
    uint8_t* dst = z + row * g.Kp + col0 + kb;
    put32(dst, re, nbytes);
    put32(dst + plane, im, nbytes);
    if (g.neg_plane) {
#pragma unroll
      for (int x = 0; x < 8; ++x) re[x] ^= 0x80808080u;
      put32(dst + 2 * plane, re, nbytes);
    }
  }
}

// [chan][pol][ant][t] source: every output row is n_seg contiguous runs of K
// bytes (one per summed pol).  One thread converts 16 columns of one row.
__global__ void __launch_bounds__(256) ftd_cpat_to_planes_kernel(const uint8_t* __restrict__ raw,
                                                                 uint8_t* __restrict__ z,
                                                                 FtdGeom g) {
  const int chunks = g.Kp >> 4;
  const int64_t total = g.rows * chunks;
  const int n_seg = g.pol_sum ? g.n_pol : 1;
  const int64_t plane = g.rows * int64_t(g.Kp);
  for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < total;
       x += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = x / chunks;
    const int c0 = int(x - row * chunks) << 4;
    const int ant = int(row % g.n_ant);
    const int64_t b = row / g.n_ant;
    const int ti = int(b % g.n_ti);
    const int64_t cp = b / g.n_ti;  // chan*n_pol + pol, or chan with pol_sum
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    const int seg = c0 / g.K, k = c0 - seg * g.K;
    if (seg < n_seg && k + 16 <= g.K) {  // one segment: contiguous source bytes
      const int64_t src_row = g.pol_sum ? ((cp * g.n_pol + seg) * g.n_ant + ant)
                                        : (cp * g.n_ant + ant);
      const uint8_t* src = raw + src_row * g.n_time + int64_t(ti) * g.K + k;
      if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(src));
        w[0] = v.x, w[1] = v.y, w[2] = v.z, w[3] = v.w;
      } else {
        for (int bb = 0; bb < 16; ++bb) w[bb >> 2] |= uint32_t(__ldg(src + bb)) << (8 * (bb & 3));
      }
    } else {
      for (int bb = 0; bb < 16; ++bb) {
        const int c = c0 + bb;
        const int sg = c / g.K, kk = c - sg * g.K;
        if (sg >= n_seg) break;
        const int64_t src_row = g.pol_sum ? ((cp * g.n_pol + sg) * g.n_ant + ant)
                                          : (cp * g.n_ant + ant);
        w[bb >> 2] |= uint32_t(__ldg(raw + src_row * g.n_time + int64_t(ti) * g.K + kk))
                      << (8 * (bb & 3));
      }
    }
    uint32_t re[4], im[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) qc4_to_e4m3(w[q], re[q], im[q]);
    uint8_t* dst = z + row * g.Kp + c0;
    *reinterpret_cast<uint4*>(dst) = make_uint4(re[0], re[1], re[2], re[3]);
    *reinterpret_cast<uint4*>(dst + plane) = make_uint4(im[0], im[1], im[2], im[3]);
    if (g.neg_plane) {
      constexpr uint32_t kS = 0x80808080u;
      *reinterpret_cast<uint4*>(dst + 2 * plane) =
          make_uint4(re[0] ^ kS, re[1] ^ kS, re[2] ^ kS, re[3] ^ kS);
    }
  }
}

}  // namespace

cudaError_t launch_ftd_to_planes(const uint8_t* raw, uint8_t* z, const FtdGeom& g, int layout,
                                 int sm_count, cudaStream_t s) {
  if (layout == 0) {
    const int64_t S = int64_t(g.n_ant) * g.n_chan * g.n_pol;
    const int kmax = g.pol_sum ? g.Kp - (g.n_pol - 1) * g.K : g.Kp;
    const dim3 grid(unsigned((S + kTS - 1) / kTS), unsigned((kmax + kTK - 1) / kTK),
                    unsigned(g.n_ti));
    if (grid.y > 65535u || grid.z > 65535u || S >= (int64_t(1) << 31))
      return cudaErrorInvalidConfiguration;
    ftd_tacp_to_planes_kernel<<<grid, 256, 0, s>>>(raw, z, g);
  } else {
    const int64_t total = g.rows * (g.Kp >> 4);
    int64_t blocks = (total + 255) / 256;
    if (blocks > int64_t(sm_count) * 16) blocks = int64_t(sm_count) * 16;
    if (blocks < 1) blocks = 1;
    ftd_cpat_to_planes_kernel<<<unsigned(blocks), 256, 0, s>>>(raw, z, g);
  }
  return cudaGetLastError();
}

}  // namespace ftdx
