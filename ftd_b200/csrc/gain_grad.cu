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
// One block per 64 x 64 tile of one channel's triangle: rows stream through
// the block coalesced (64 consecutive packed elements per row segment), row
// sums are warp-reduced, column sums stay in registers, and each block adds
// its 128 partial gradients and its loss to FP64 accumulators with atomics.
#include <cstdint>

#include "herk_fp8.cuh"

namespace ftdx {
namespace {

constexpr int kGT = 64;  // tile edge

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

  __shared__ float2 gi[kGT], gj[kGT];
  __shared__ double col_re[4][kGT], col_im[4][kGT];
  __shared__ double row_re[kGT], row_im[kGT];
  __shared__ double lsum[8];
  const int tid = threadIdx.x;
  if (tid < kGT) {
    gi[tid] = (i0 + tid < n) ? g[i0 + tid] : make_float2(0.f, 0.f);
    gj[tid] = (j0 + tid < n) ? g[j0 + tid] : make_float2(0.f, 0.f);
  }
  __syncthreads();

  const int cl = tid & 63;  // column within the tile (fixed per thread)
  const int rg = tid >> 6;  // row group 0..3
  const int j = j0 + cl;
  double cre = 0.0, cim = 0.0, lacc = 0.0;
  for (int rr = rg; rr < kGT; rr += 4) {
    const int i = i0 + rr;
    float rre = 0.f, rim = 0.f;
    if (i < n && j <= i) {
      const int64_t e = int64_t(i) * (i + 1) / 2 + j;
      const float2 o = __ldcs(ro + e), m0 = __ldcs(rm + e);
      const float wt = __ldcs(wc + e);
      const float2 a = gi[rr], b = gj[cl];
      // M = g_i * R_mod * conj(g_j)
      const float tr = a.x * m0.x - a.y * m0.y, tim = a.x * m0.y + a.y * m0.x;
      const float mr = tr * b.x + tim * b.y, mi = tim * b.x - tr * b.y;
      const float er = o.x - mr, ei = o.y - mi;
      const double mult = (i == j) ? 1.0 : 2.0;
      lacc += mult * double(wt) * (double(er) * er + double(ei) * ei);
      // c = W E conj(R_mod)
      const float cr = wt * (er * m0.x + ei * m0.y), ci = wt * (ei * m0.x - er * m0.y);
      // row i gets c g_j; column j gets conj(c) g_i (not for the diagonal)
      rre = cr * b.x - ci * b.y;
      rim = cr * b.y + ci * b.x;
      if (i != j) {
        cre += double(cr * a.x + ci * a.y);
        cim += double(cr * a.y - ci * a.x);
      }
    }
    // reduce the row over the 64 threads sharing it (two warps)
    double dre = rre, dim = rim;
    for (int o = 16; o > 0; o >>= 1) {
      dre += __shfl_xor_sync(0xffffffffu, dre, o);
      dim += __shfl_xor_sync(0xffffffffu, dim, o);
    }
    // lanes 0 of the two warps of this row group combine through shared memory
    if ((tid & 31) == 0) {
      if ((tid & 63) == 0) {
        row_re[rr] = dre;
        row_im[rr] = dim;
      }
    }
    __syncthreads();
    if ((tid & 63) == 32) {
      row_re[rr] += dre;
      row_im[rr] += dim;
    }
    __syncthreads();
  }
  col_re[rg][cl] = cre;
  col_im[rg][cl] = cim;
  for (int o = 16; o > 0; o >>= 1) lacc += __shfl_xor_sync(0xffffffffu, lacc, o);
  if ((tid & 31) == 0) lsum[tid >> 5] = lacc;
  __syncthreads();
  if (tid < kGT) {
    const int i = i0 + tid;
    if (i < n) {
      atomicAdd(grad + 2 * i, -4.0 * row_re[tid]);
      atomicAdd(grad + 2 * i + 1, -4.0 * row_im[tid]);
    }
  } else if (tid < 2 * kGT) {
    const int c = tid - kGT;
    const int jj = j0 + c;
    if (jj < n) {
      const double sre = col_re[0][c] + col_re[1][c] + col_re[2][c] + col_re[3][c];
      const double sim = col_im[0][c] + col_im[1][c] + col_im[2][c] + col_im[3][c];
      atomicAdd(grad + 2 * jj, -4.0 * sre);
      atomicAdd(grad + 2 * jj + 1, -4.0 * sim);
    }
  } else if (tid == 2 * kGT) {
    double s = 0.0;
    for (int k = 0; k < 8; ++k) s += lsum[k];
    atomicAdd(loss, s);
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
