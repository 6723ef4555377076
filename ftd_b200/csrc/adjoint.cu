// adjoint.cu -- adjoint of the correlator: dV = (G + G^H) V per channel.
//
// For a loss L(R) of the visibilities R = V V^H with upstream gradient
// G = dL/dR (N x N complex per channel), the gradient with respect to the
// voltages is (G + G^H) V.  V is QC int4 (exact in bf16); G is complex64, so
// S = G + G^H is split into bf16 hi + lo parts (S = S_hi + S_lo with
// |S_lo| <= 2^-8 |S|, residual error ~2^-16 relative) and
//   dV = S_hi V + S_lo V
// runs on the tensor cores (tcgen05.mma kind::f16, FP32 accumulation).
//
//  * sym_split_kernel: S = G + G^H, one block per pair of mirrored 32 x 32
//    tiles (each element of G read once), written as four bf16 planes Re_hi,
//    Im_hi, Re_lo, Im_lo [batch*N][N].
//  * vt_kernel: V [batch][N][K] QC -> V^T planes Re, Im [batch*K][N] bf16.
//  * adjoint_tc_kernel: persistent; tile = 128 time samples (MMA M) x 128
//    antennas (MMA N), K = antennas contracted, 2-stage TMA ring of six
//    128 x 64 bf16 planes; per 16-antenna k-step eight MMAs:
//      Re += Vr Sr_X - Vi Si_X,  Im += Vr Si_X + Vi Sr_X   (X = hi, lo)
//    into a double-buffered Re | Im accumulator; the epilogue stores dV[a][t]
//    with a warp's 32 lanes on 32 consecutive t (256-byte coalesced rows).
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "herk_fp8.cuh"
#include "sm100.cuh"

namespace ftdx {
using namespace dev;
namespace {

constexpr int kAT = 128;                        // tile edge (t and a)
constexpr int kAK = 64;                         // antennas per stage (128 B of bf16)
constexpr int kAPlane = kAT * kAK * 2;          // 16 KB
constexpr int kANumPlanes = 6;                  // Vr, Vi, Sr_hi, Si_hi, Sr_lo, Si_lo
constexpr int kAStageBytes = kANumPlanes * kAPlane;
constexpr int kAStages = 2;
constexpr int kAThreads = 192;                  // TMA warp, MMA warp, 4 epilogue warps
constexpr size_t kASmem = 1024 + size_t(kAStages) * kAStageBytes + 256;

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// S = G + G^H, one block per pair of mirrored 32 x 32 tiles (tile row i >=
// tile column j, 16 x 16 threads): the block reads G's tiles (i, j) and
// (j, i) once each -- every element of G crosses HBM once -- and writes S's
// tiles (i, j) and (j, i):  S[a][c] = G[a][c] + conj(G[c][a]).  Thread (x, y)
// owns rows y, y + 16 and columns 2x, 2x + 1 of a tile: its two elements of
// a row arrive as one 16-byte load when G is 16-byte aligned, and each bf16
// plane is written in pairs.  n is a multiple of 8, so tiles never straddle
// the matrix edge by an odd column.
__device__ __forceinline__ float4 load2(const float2* p, bool v16) {
  if (v16) return __ldcs(reinterpret_cast<const float4*>(p));
  const float2 u = __ldcs(p), v = __ldcs(p + 1);
  return make_float4(u.x, u.y, v.x, v.y);
}

__global__ void __launch_bounds__(256) sym_split_kernel(const float2* __restrict__ G,
                                                        __nv_bfloat16* __restrict__ S, int n,
                                                        int64_t plane_elems) {
  __shared__ float2 tile[2][32][33];  // [0] = G tile (i, j), [1] = G tile (j, i)
  const int b = blockIdx.y;
  const int r = blockIdx.x;  // lower-triangle tile index -> (ti, tj), tj <= ti
  int ti = int((sqrtf(8.f * float(r) + 1.f) - 1.f) * 0.5f);
  while (ti > 0 && ti * (ti + 1) / 2 > r) --ti;
  while ((ti + 1) * (ti + 2) / 2 <= r) ++ti;
  const int tj = r - ti * (ti + 1) / 2;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const float2* Gb = G + int64_t(b) * n * n;
  const bool v16 = (reinterpret_cast<uintptr_t>(G) & 15) == 0;
  const int nt = ti == tj ? 1 : 2;
  // loads: both tiles, rows ty and ty + 16, columns 2 tx, 2 tx + 1
  float4 v[2][2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int rb = (q == 0 ? ti : tj) * 32, cb = (q == 0 ? tj : ti) * 32;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int a = rb + ty + 16 * k, c = cb + 2 * tx;
      v[q][k] = (q < nt && a < n && c < n) ? load2(Gb + int64_t(a) * n + c, v16)
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      tile[q][ty + 16 * k][2 * tx] = make_float2(v[q][k].x, v[q][k].y);
      tile[q][ty + 16 * k][2 * tx + 1] = make_float2(v[q][k].z, v[q][k].w);
    }
  __syncthreads();
  // S tile (i, j) from tile[0] and the transpose of tile[1]; S tile (j, i)
  // from tile[1] and the transpose of tile[0] (a diagonal tile: itself)
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (q >= nt) break;
    const int rb = (q == 0 ? ti : tj) * 32, cb = (q == 0 ? tj : ti) * 32;
    const int other = nt == 1 ? 0 : 1 - q;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int rl = ty + 16 * k, a = rb + rl, c = cb + 2 * tx;
      if (a >= n || c >= n) continue;
      const float2 g0 = tile[q][rl][2 * tx], g1 = tile[q][rl][2 * tx + 1];
      const float2 t0 = tile[other][2 * tx][rl], t1 = tile[other][2 * tx + 1][rl];
      const float sr0 = g0.x + t0.x, si0 = g0.y - t0.y;
      const float sr1 = g1.x + t1.x, si1 = g1.y - t1.y;
      __nv_bfloat16 rh0, rl0, ih0, il0, rh1, rl1, ih1, il1;
      split_bf16(sr0, rh0, rl0);
      split_bf16(si0, ih0, il0);
      split_bf16(sr1, rh1, rl1);
      split_bf16(si1, ih1, il1);
      const int64_t o = (int64_t(b) * n + a) * n + c;
      *reinterpret_cast<__nv_bfloat162*>(S + o) = __halves2bfloat162(rh0, rh1);
      *reinterpret_cast<__nv_bfloat162*>(S + plane_elems + o) = __halves2bfloat162(ih0, ih1);
      *reinterpret_cast<__nv_bfloat162*>(S + 2 * plane_elems + o) = __halves2bfloat162(rl0, rl1);
      *reinterpret_cast<__nv_bfloat162*>(S + 3 * plane_elems + o) = __halves2bfloat162(il0, il1);
    }
  }
}

// V^T planes: VT[p][b*K + t][a] = Re/Im of V[b][a][t] (QC sign-magnitude).
__global__ void vt_kernel(const uint8_t* __restrict__ V, __nv_bfloat16* __restrict__ VT, int n,
                          int K, int64_t plane_elems) {
  __shared__ uint8_t tt[32][33];
  const int b = blockIdx.z;
  const int t0 = blockIdx.y * 32, a0 = blockIdx.x * 32;
  const uint8_t* Vb = V + int64_t(b) * n * K;
  for (int y = threadIdx.y; y < 32; y += 8) {
    const int a = a0 + y, t = t0 + threadIdx.x;
    tt[y][threadIdx.x] = (a < n && t < K) ? Vb[int64_t(a) * K + t] : uint8_t(0);
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += 8) {
    const int t = t0 + y, a = a0 + threadIdx.x;
    if (t >= K || a >= n) continue;
    const uint8_t q = tt[threadIdx.x][y];
    const int hr = (q >> 4) & 7, lr = q & 7;
    const float re = (q & 0x80) ? -float(hr) : float(hr);
    const float im = (q & 0x08) ? -float(lr) : float(lr);
    const int64_t o = (int64_t(b) * K + t) * n + a;
    VT[o] = __float2bfloat16_rn(re);
    VT[plane_elems + o] = __float2bfloat16_rn(im);
  }
}

struct AdjArgs {
  int n, K, batch;
  int tiles_t, tiles_a;   // per channel
  int num_tiles;
  float2* out;            // dV [batch][n][K]
  uint32_t* status;
};

__global__ void __launch_bounds__(kAThreads, 1)
    adjoint_tc_kernel(const __grid_constant__ CUtensorMap tmV, const __grid_constant__ CUtensorMap tmS,
                      const AdjArgs args) {
  extern __shared__ uint8_t smem_dyn[];
  uint8_t* smem = smem_dyn + ((1024u - (smem_u32(smem_dyn) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kAStages * kAStageBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kAStages + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const uint32_t smem0 = smem_u32(smem);
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (kAStages + s); };
  auto tfull_bar = [&](int b) { return bar0 + 8u * (2 * kAStages + b); };
  auto tempty_bar = [&](int b) { return bar0 + 8u * (2 * kAStages + 2 + b); };
  const uint32_t done_bar = bar0 + 8u * (2 * kAStages + 4);
  auto plane = [&](int s, int p) { return smem0 + uint32_t(s * kAStageBytes + p * kAPlane); };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kAStages; ++s) {
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
    tma_prefetch_desc(&tmV);
    tma_prefetch_desc(&tmS);
  }
  if (warp == 1) {
    tmem_alloc(smem_u32(tmem_slot), 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int per_chan = args.tiles_t * args.tiles_a;
  const int kblocks = (args.n + kAK - 1) / kAK;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0, issued = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
        const int ch = t / per_chan, r = t - ch * per_chan;
        const int tt = r / args.tiles_a, ta = r - tt * args.tiles_a;
        const int32_t rowV = ch * args.K + tt * kAT;   // V^T rows (time)
        const int32_t rowS = ch * args.n + ta * kAT;   // S rows (antennas a)
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutProducer);
            ok = false;
            break;
          }
          const int32_t k0 = kb * kAK;
          mbar_arrive_expect_tx(full_bar(stage), kAStageBytes);
          tma_load_3d(plane(stage, 0), &tmV, k0, rowV, 0, full_bar(stage));
          tma_load_3d(plane(stage, 1), &tmV, k0, rowV, 1, full_bar(stage));
          for (int p = 0; p < 4; ++p)
            tma_load_3d(plane(stage, 2 + p), &tmS, k0, rowS, p, full_bar(stage));
          ++issued;
          if (++stage == kAStages) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) {
        int s = stage;
        uint32_t ph = phase;
        for (int q = 0; q < kAStages && q < issued; ++q) {
          if (--s < 0) {
            s = kAStages - 1;
            ph ^= 1u;
          }
          volatile int never = 0;
          if (!mbar_wait(full_bar(s), ph, &never)) atomicOr(args.status, kStatusTimeoutOther);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_f32acc(1, 1, kAT, kAT);      // bf16 x bf16
      constexpr uint32_t idesc_neg = idesc_f32acc(1, 1, kAT, kAT, 1);
      int stage = 0, acc = 0;
      uint32_t phase = 0, acc_phase = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < args.num_tiles && ok; t += gridDim.x) {
        if (!mbar_wait(tempty_bar(acc), acc_phase ^ 1u, abort_flag)) {
          atomicOr(args.status, kStatusTimeoutMma);
          break;
        }
        tc_fence_after();
        const uint32_t d_re = tmem_base + uint32_t(acc * 2 * kAT);
        const uint32_t d_im = d_re + uint32_t(kAT);
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait(full_bar(stage), phase, abort_flag)) {
            atomicOr(args.status, kStatusTimeoutMma);
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int s = 0; s < (kAK * 2) / 32; ++s) {  // 16 antennas (32 B) per k-step
            const uint64_t vr = sdesc_sw128_kmajor(plane(stage, 0) + 32 * s);
            const uint64_t vi = sdesc_sw128_kmajor(plane(stage, 1) + 32 * s);
            const uint32_t first = (kb | s) != 0;
#pragma unroll
            for (int x = 0; x < 2; ++x) {  // hi, lo
              const uint64_t sr = sdesc_sw128_kmajor(plane(stage, 2 + 2 * x) + 32 * s);
              const uint64_t si = sdesc_sw128_kmajor(plane(stage, 3 + 2 * x) + 32 * s);
              mma_f16(d_re, vr, sr, idesc, x == 0 ? first : 1u);
              mma_f16(d_im, vr, si, idesc, x == 0 ? first : 1u);
              mma_f16(d_re, vi, si, idesc_neg, 1);
              mma_f16(d_im, vi, sr, idesc, 1);
            }
          }
          mma_commit(empty_bar(stage));
          if (++stage == kAStages) {
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
    const int q = warp & 3;
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int t = blockIdx.x; t < args.num_tiles; t += gridDim.x) {
      const int ch = t / per_chan, r = t - ch * per_chan;
      const int tt = r / args.tiles_a, ta = r - tt * args.tiles_a;
      const bool ok = __all_sync(0xffffffffu, mbar_wait(tfull_bar(acc), acc_phase, abort_flag));
      if (!ok) {
        if (lane == 0) atomicOr(args.status, kStatusTimeoutEpilogue);
        break;
      }
      tc_fence_after();
      const int tsamp = tt * kAT + q * 32 + lane;  // this lane's time sample
      const uint32_t tb = tmem_base + (uint32_t(q * 32) << 16) + uint32_t(acc * 2 * kAT);
      float2* outc = args.out + int64_t(ch) * args.n * args.K;
#pragma unroll 1
      for (int c = 0; c < kAT / 32; ++c) {
        const int a0 = ta * kAT + 32 * c;
        if (a0 >= args.n) continue;
        uint32_t re[32], im[32];
        __syncwarp();
        tmem_ld_32x32b_x32(tb + 32u * c, re);
        tmem_ld_32x32b_x32(tb + uint32_t(kAT) + 32u * c, im);
        tmem_wait_ld();
        if (tsamp < args.K) {
#pragma unroll
          for (int m = 0; m < 32; ++m) {
            const int a = a0 + m;
            if (a < args.n)
              __stcs(outc + int64_t(a) * args.K + tsamp,
                     make_float2(__uint_as_float(re[m]), __uint_as_float(im[m])));
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
    tmem_dealloc(tmem_base, 512);
  }
}

}  // namespace

size_t adjoint_workspace_bytes(int n, int K, int batch) {
  const size_t s_planes = 4 * size_t(batch) * n * n * 2;
  const size_t v_planes = 2 * size_t(batch) * K * n * 2;
  return s_planes + v_planes + 1024;
}

cudaError_t launch_adjoint(const void* G, const uint8_t* V, void* dV, int n, int K, int batch,
                           uint8_t* ws, int sm_count, uint32_t* status, void* encode_fn,
                           cudaStream_t s) {
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(encode_fn);
  if (!encode) return cudaErrorInvalidValue;
  const int64_t s_plane = int64_t(batch) * n * n;
  const int64_t v_plane = int64_t(batch) * K * n;
  __nv_bfloat16* S = reinterpret_cast<__nv_bfloat16*>(ws);
  __nv_bfloat16* VT = reinterpret_cast<__nv_bfloat16*>(
      ws + ((4 * size_t(s_plane) * 2 + 1023) / 1024) * 1024);
  const int nt = (n + 31) / 32;
  sym_split_kernel<<<dim3(unsigned(nt * (nt + 1) / 2), unsigned(batch)), dim3(16, 16), 0, s>>>(
      static_cast<const float2*>(G), S, n, s_plane);
  const dim3 tb(32, 8);
  vt_kernel<<<dim3((n + 31) / 32, (K + 31) / 32, batch), tb, 0, s>>>(V, VT, n, K, v_plane);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;

  CUtensorMap tmV, tmS;
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint32_t box[3] = {cuuint32_t(kAK), cuuint32_t(kAT), 1};
  {
    const cuuint64_t dims[3] = {cuuint64_t(n), cuuint64_t(int64_t(batch) * K), 2};
    const cuuint64_t str[2] = {cuuint64_t(n) * 2, cuuint64_t(v_plane) * 2};
    if (encode(&tmV, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, VT, dims, str, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
  }
  {
    const cuuint64_t dims[3] = {cuuint64_t(n), cuuint64_t(int64_t(batch) * n), 4};
    const cuuint64_t str[2] = {cuuint64_t(n) * 2, cuuint64_t(s_plane) * 2};
    if (encode(&tmS, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, S, dims, str, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
  }
  AdjArgs a;
  a.n = n;
  a.K = K;
  a.batch = batch;
  a.tiles_t = (K + kAT - 1) / kAT;
  a.tiles_a = (n + kAT - 1) / kAT;
  a.num_tiles = batch * a.tiles_t * a.tiles_a;
  a.out = static_cast<float2*>(dV);
  a.status = status;
  e = ensure_smem_limit(reinterpret_cast<const void*>(adjoint_tc_kernel), kASmem);
  if (e != cudaSuccess) return e;
  const int grid = a.num_tiles < sm_count ? a.num_tiles : sm_count;
  adjoint_tc_kernel<<<grid, kAThreads, kASmem, s>>>(tmV, tmS, a);
  return cudaGetLastError();
}

}  // namespace ftdx
