// gain_grad.cu -- loss and gradient of gain calibration on packed triangles.
//
// For per-input complex gains g (shared by all channels), observed and model
// visibilities R_obs, R_mod and real weights W (all packed lower triangles,
// Hermitian, one per channel):
//   M_ij = g_i R_mod,ij conj(g_j),   E_ij = R_obs,ij - M_ij
//   L    = sum_f sum_{i,j} W_ij |E_ij|^2          (full matrices: off-diagonal
//                                                 entries of the triangle count twice)
//   grad_k = dL/dRe(g_k) + i dL/dIm(g_k) = 2 dL/dconj(g_k)
//          = -4 sum_f sum_j W_kj E_kj conj(R_mod,kj) g_j
// For a stored element (i, j < i), c = W E_ij conj(R_mod,ij) feeds row i
// through c g_j and row j through conj(c) g_i (the Hermitian mirror).
//
// One block per 64 x 64 tile of one channel's triangle.  Warp w owns rows w,
// w + 8, ... of the tile and lane l its columns 2l, 2l + 1, so a row segment
// (64 consecutive packed elements) is one coalesced warp load and its sum a
// warp reduction, with no block barrier per row; two rows' loads are in
// flight per lane.  Column sums stay in registers until one shared-memory
// combine per tile.  Within a tile the partial sums are FP32 (at most 64
// terms); across tiles they are added to FP64 accumulators with atomics, and
// the loss is accumulated in FP64.
#include <cstdint>

#include "herk_fp8.cuh"

namespace ftdx {
namespace {

constexpr int kGT = 64;         // tile edge
constexpr int kGWarps = 8;      // rows of a tile are dealt to 8 warps

struct GainTerms {
  float rre, rim;   // row i's contribution c g_j
  float cre, cim;   // column j's contribution conj(c) g_i (zero on the diagonal)
  double l;         // W |E|^2 (times 2 off the diagonal)
};

__device__ __forceinline__ GainTerms gain_terms(float2 o, float2 m0, float wt, float2 a, float2 b,
                                                bool diag) {
  // M = g_i R_mod conj(g_j), E = R_obs - M, c = W E conj(R_mod)
  const float tr = a.x * m0.x - a.y * m0.y, tim = a.x * m0.y + a.y * m0.x;
  const float mr = tr * b.x + tim * b.y, mi = tim * b.x - tr * b.y;
  const float er = o.x - mr, ei = o.y - mi;
  const float cr = wt * (er * m0.x + ei * m0.y), ci = wt * (ei * m0.x - er * m0.y);
  GainTerms t;
  t.rre = cr * b.x - ci * b.y;
  t.rim = cr * b.y + ci * b.x;
  t.cre = diag ? 0.f : cr * a.x + ci * a.y;
  t.cim = diag ? 0.f : cr * a.y - ci * a.x;
  t.l = (diag ? 1.0 : 2.0) * double(wt) * (double(er) * er + double(ei) * ei);
  return t;
}

__global__ void __launch_bounds__(256) gain_grad_kernel(const float2* __restrict__ robs,
                                                        const float2* __restrict__ rmod,
                                                        const float* __restrict__ w,
                                                        const float2* __restrict__ g, int n,
                                                        int tiles_per_chan,
                                                        double* __restrict__ grad,  // [n][2]
                                                        double* __restrict__ loss) {
  const int ch = blockIdx.y;
  // tile (ti, tj), tj <= ti, from the linear index
  const int r = blockIdx.x;
  if (r >= tiles_per_chan) return;
  int ti = int((sqrtf(8.f * float(r) + 1.f) - 1.f) * 0.5f);
  while (ti > 0 && ti * (ti + 1) / 2 > r) --ti;
  while ((ti + 1) * (ti + 2) / 2 <= r) ++ti;
  const int tj = r - ti * (ti + 1) / 2;
  const int i0 = ti * kGT, j0 = tj * kGT;
  const int64_t P = int64_t(n) * (n + 1) / 2;
  const float2* ro = robs + int64_t(ch) * P;
  const float2* rm = rmod + int64_t(ch) * P;
  const float* wc = w + int64_t(ch) * P;

  __shared__ float2 gi[kGT];
  __shared__ float row_re[kGT], row_im[kGT];
  __shared__ float col_re[kGWarps][kGT], col_im[kGWarps][kGT];
  __shared__ double lsum[kGWarps];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid < kGT) gi[tid] = (i0 + tid < n) ? g[i0 + tid] : make_float2(0.f, 0.f);
  // this lane's two columns and their gains
  const int j[2] = {j0 + 2 * lane, j0 + 2 * lane + 1};
  float2 gj[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) gj[c] = j[c] < n ? __ldg(g + j[c]) : make_float2(0.f, 0.f);
  __syncthreads();

  float cre[2] = {0.f, 0.f}, cim[2] = {0.f, 0.f};
  double lacc = 0.0;
  // rows warp, warp + 8, ...: two rows per iteration (loads of both issued first)
#pragma unroll 1
  for (int rr = warp; rr < kGT; rr += 2 * kGWarps) {
    float2 o[2][2], m[2][2];
    float wt[2][2];
    bool ok[2][2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = i0 + rr + h * kGWarps;
      const int64_t e0 = int64_t(i) * (i + 1) / 2;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        ok[h][c] = i < n && j[c] <= i;
        o[h][c] = ok[h][c] ? __ldcs(ro + e0 + j[c]) : make_float2(0.f, 0.f);
        m[h][c] = ok[h][c] ? __ldcs(rm + e0 + j[c]) : make_float2(0.f, 0.f);
        wt[h][c] = ok[h][c] ? __ldcs(wc + e0 + j[c]) : 0.f;
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = rr + h * kGWarps, i = i0 + row;
      const float2 a = gi[row];
      float rre = 0.f, rim = 0.f;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (!ok[h][c]) continue;
        const GainTerms t = gain_terms(o[h][c], m[h][c], wt[h][c], a, gj[c], i == j[c]);
        rre += t.rre;
        rim += t.rim;
        cre[c] += t.cre;
        cim[c] += t.cim;
        lacc += t.l;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        rre += __shfl_xor_sync(0xffffffffu, rre, off);
        rim += __shfl_xor_sync(0xffffffffu, rim, off);
      }
      if (lane == 0) {
        row_re[row] = rre;
        row_im[row] = rim;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    col_re[warp][2 * lane + c] = cre[c];
    col_im[warp][2 * lane + c] = cim[c];
  }
  for (int off = 16; off > 0; off >>= 1) lacc += __shfl_xor_sync(0xffffffffu, lacc, off);
  if (lane == 0) lsum[warp] = lacc;
  __syncthreads();
  if (tid < kGT) {
    const int i = i0 + tid;
    if (i < n) {
      atomicAdd(grad + 2 * i, -4.0 * double(row_re[tid]));
      atomicAdd(grad + 2 * i + 1, -4.0 * double(row_im[tid]));
    }
  } else if (tid < 2 * kGT) {
    const int c = tid - kGT;
    const int jj = j0 + c;
    if (jj < n) {
      float sre = 0.f, sim = 0.f;
#pragma unroll
      for (int q = 0; q < kGWarps; ++q) {
        sre += col_re[q][c];
        sim += col_im[q][c];
      }
      atomicAdd(grad + 2 * jj, -4.0 * double(sre));
      atomicAdd(grad + 2 * jj + 1, -4.0 * double(sim));
    }
  } else if (tid == 2 * kGT) {
    double sacc = 0.0;
    for (int q = 0; q < kGWarps; ++q) sacc += lsum[q];
    atomicAdd(loss, sacc);
  }
}

}  // namespace

cudaError_t launch_gain_grad(const float2* robs, const float2* rmod, const float* w,
                             const float2* g, int n, int nchan, double* grad, double* loss,
                             cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(grad, 0, sizeof(double) * 2 * size_t(n), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(loss, 0, sizeof(double), s);
  if (e != cudaSuccess) return e;
  const int nt = (n + kGT - 1) / kGT;
  const int per = nt * (nt + 1) / 2;
  gain_grad_kernel<<<dim3(unsigned(per), unsigned(nchan)), 256, 0, s>>>(robs, rmod, w, g, n, per,
                                                                       grad, loss);
  return cudaGetLastError();
}

}  // namespace ftdx
