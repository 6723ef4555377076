// imaging.cu -- UV gridding of the packed triangles with fused polarisation
// reduction and taper, inverse 2-D FFT (cuFFT), beam extraction
// (ftdx_image_beams).  Replaces the FP32 paths of
// imaging_pipeline::ImagingPipeline::grid_and_image (lib/imaging_pipeline.cu)
// and stages 2-5 of VisibilityBeamformer::compute (lib/visibility_bf.cpp:305-380);
// cell arithmetic as uv_cell / pillbox_grid_scatter_fp32_fp32grid_kernel
// (include/kernels/imaging_kernels.cuh:37-47, 219-268).
#include <cufft.h>

#include <climits>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>

#include "context.h"

namespace ftdx {

struct ImagingState {
  float2* grid = nullptr;
  size_t grid_bytes = 0;
  std::map<std::pair<int, int>, cufftHandle> plans;  // (Ng, channels) -> plan
  void* sort = nullptr;  // beam pixel keys / indices (in, sorted) + radix-sort scratch
  size_t sort_bytes = 0;
  ~ImagingState() {
    for (auto& p : plans) cufftDestroy(p.second);
    if (grid) cudaFree(grid);
    if (sort) cudaFree(sort);
  }
};

// Beam lists at least this long are gathered in pixel order.
constexpr int kSortedBeams = 65536;

namespace {

constexpr double kLightSpeed = 299792458.0;

// Row i and column j of packed lower-triangle index k = i(i+1)/2 + j: a float
// square-root estimate, corrected in integers (exact for every k).
__device__ __forceinline__ void tri_row_col(int64_t k, int& i, int& j) {
  int64_t r = int64_t((sqrtf(8.f * float(k) + 1.f) - 1.f) * 0.5f);
  while (r * (r + 1) / 2 > k) --r;
  while ((r + 1) * (r + 2) / 2 <= k) ++r;
  i = int(r);
  j = int(k - r * (r + 1) / 2);
}

constexpr int kMaxTileChans = 64;  // channels of one grid tile (wavelengths in shared memory)

// One thread per baseline, looping over the tile's channels: sum the n_pol
// visibilities, then add them (times the taper weight of the cell) at the
// baseline's cell and, for a cross-correlation, the conjugate at the
// mirrored cell.  The baseline's (u, v) and its row / column are read and
// decoded once per tile; the wavelengths sit in shared memory.  Only cells in
// grid rows [r0, r1) are written: a grid too large for L2 is scattered in
// row bands (one launch each), so that every atomic resolves in L2.
__global__ void __launch_bounds__(256) grid_scatter_kernel(
    const float2* __restrict__ vis, const float2* __restrict__ uv, const double* __restrict__ freq,
    const float* __restrict__ taper, float2* __restrict__ grid, int64_t n_bl, int n_pol, int Ng,
    int f0, int nf, float cell, int r0, int r1) {
  __shared__ double lambda[kMaxTileChans];
  for (int f = threadIdx.x; f < nf; f += blockDim.x) lambda[f] = kLightSpeed / freq[f0 + f];
  __syncthreads();
  const int64_t plane = int64_t(Ng) * Ng;
  const float half = 0.5f * float(Ng);
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n_bl;
       k += int64_t(gridDim.x) * blockDim.x) {
    const float2 b = __ldg(uv + k);
    int i, j;
    tri_row_col(k, i, j);
    const bool cross = i != j;
    for (int fl = 0; fl < nf; ++fl) {
      const float2* vp = vis + int64_t(f0 + fl) * n_pol * n_bl + k;
      float2 v = __ldg(vp);
      for (int p = 1; p < n_pol; ++p) {
        const float2 w = __ldg(vp + int64_t(p) * n_bl);
        v.x += w.x;
        v.y += w.y;
      }
      const double lam = lambda[fl];
      const float ul = float(double(b.x) / lam), vl = float(double(b.y) / lam);
      float2* g = grid + int64_t(fl) * plane;
      const int iu = int(roundf(ul / cell + half)), iv = int(roundf(vl / cell + half));
      if (iu >= 0 && iu < Ng && iv >= r0 && iv < r1) {
        const int64_t c = int64_t(iv) * Ng + iu;
        const float wt = taper ? __ldg(taper + c) : 1.f;
        atomicAdd(g + c, make_float2(v.x * wt, v.y * wt));
      }
      if (cross) {
        const int iuc = int(roundf(-ul / cell + half)), ivc = int(roundf(-vl / cell + half));
        if (iuc >= 0 && iuc < Ng && ivc >= r0 && ivc < r1) {
          const int64_t c = int64_t(ivc) * Ng + iuc;
          const float wt = taper ? __ldg(taper + c) : 1.f;
          atomicAdd(g + c, make_float2(v.x * wt, -v.y * wt));
        }
      }
    }
  }
}

__global__ void beam_extract_kernel(const float2* __restrict__ img, const int* __restrict__ pix,
                                    float* __restrict__ beams, int Ng, int n_beam, int nf,
                                    float norm) {
  const int total = nf * n_beam;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < total; x += gridDim.x * blockDim.x) {
    const int fl = x / n_beam, b = x - fl * n_beam;
    const int r = __ldg(pix + 2 * b), c = __ldg(pix + 2 * b + 1);
    float out = 0.f;
    if (r >= 0 && r < Ng && c >= 0 && c < Ng) {
      const float2 z = img[int64_t(fl) * Ng * Ng + int64_t(r) * Ng + c];
      out = (z.x * z.x + z.y * z.y) * norm;
    }
    beams[x] = out;
  }
}

// Sort keys of the beam pixels: the linear pixel r * Ng + c (INT_MAX for a
// pixel outside the image, which reads as 0), value = the beam's index.
__global__ void beam_keys_kernel(const int* __restrict__ pix, int n_beam, int Ng,
                                 int* __restrict__ keys, int* __restrict__ idx) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n_beam; b += gridDim.x * blockDim.x) {
    const int r = __ldg(pix + 2 * b), c = __ldg(pix + 2 * b + 1);
    keys[b] = (r >= 0 && r < Ng && c >= 0 && c < Ng) ? r * Ng + c : INT_MAX;
    idx[b] = b;
  }
}

// Beam extraction over the pixel-sorted list: the image (larger than L2 at
// Ng = 4096) is read in address order, the results written back to each
// beam's place (the per-channel beam row stays in L2).
__global__ void beam_extract_sorted_kernel(const float2* __restrict__ img,
                                           const int* __restrict__ keys,
                                           const int* __restrict__ idx, float* __restrict__ beams,
                                           int64_t plane, int n_beam, int nf, float norm) {
  const int64_t total = int64_t(nf) * n_beam;
  for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < total;
       x += int64_t(gridDim.x) * blockDim.x) {
    const int fl = int(x / n_beam), k = int(x - int64_t(fl) * n_beam);
    const int key = __ldg(keys + k);
    float out = 0.f;
    if (key != INT_MAX) {
      const float2 z = img[int64_t(fl) * plane + key];
      out = (z.x * z.x + z.y * z.y) * norm;
    }
    beams[int64_t(fl) * n_beam + __ldg(idx + k)] = out;
  }
}

}  // namespace
}  // namespace ftdx

using namespace ftdx;

extern "C" ftdx_status ftdx_image_beams(ftdx_handle h, const ftdx_imaging_config* cfg,
                                        const void* vis, float* beams, void* grid_out,
                                        void* stream) {
  if (!h) return FTDX_ERR_INVALID_ARG;
  if (!cfg || !vis) return fail(h, FTDX_ERR_INVALID_ARG, "image_beams: null config or vis");
  const ftdx_imaging_config& c = *cfg;
  if (c.n_ant < 1 || c.n_chan < 1 || c.n_pol < 1 || c.n_grid < 2 || c.n_beam < 0 ||
      c.chan_tile < 0 || !(c.cell_size_rad > 0.f) || !c.baseline_uv_m || !c.freq_hz ||
      c.output_stage < 0 || c.output_stage > 2 || c.n_grid > 32768)
    return fail(h, FTDX_ERR_INVALID_ARG, "image_beams: bad configuration");
  if (c.output_stage == 0 && c.n_beam > 0 && (!beams || !c.beam_pixels))
    return fail(h, FTDX_ERR_INVALID_ARG, "image_beams: beams need beam_pixels and an output");
  if (c.output_stage > 0 && !grid_out)
    return fail(h, FTDX_ERR_INVALID_ARG, "image_beams: output_stage %d needs grid_out",
                c.output_stage);
  if (((reinterpret_cast<uintptr_t>(vis) | reinterpret_cast<uintptr_t>(c.baseline_uv_m)) & 7) != 0)
    return fail(h, FTDX_ERR_INVALID_ARG, "image_beams: vis and baseline_uv_m must be 8-byte aligned");
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int Ng = c.n_grid;
  const int64_t plane = int64_t(Ng) * Ng;
  const int64_t n_bl = int64_t(c.n_ant) * (c.n_ant + 1) / 2;
  int tile = c.chan_tile;
  if (tile == 0) tile = int(std::max<int64_t>(1, (int64_t(64) << 20) / (plane * 8)));
  tile = std::min(std::min(tile, c.n_chan), kMaxTileChans);
  if (!h->imaging) h->imaging = std::make_shared<ImagingState>();
  auto* st = static_cast<ImagingState*>(h->imaging.get());
  const size_t need = size_t(tile) * size_t(plane) * sizeof(float2);
  if (st->grid_bytes < need) {
    if (stream_capturing(s))
      return fail(h, FTDX_ERR_CAPACITY, "image_beams: grid workspace needed while capturing");
    cudaStreamSynchronize(s);
    if (st->grid) cudaFree(st->grid);
    st->grid = nullptr;
    st->grid_bytes = 0;
    e = cudaMalloc(&st->grid, need);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(h, FTDX_ERR_ALLOC, "image_beams: grid workspace of %zu bytes", need);
    }
    st->grid_bytes = need;
  }
  const float norm = 1.f / (float(Ng) * float(Ng));
  // long beam lists: sort the pixels once per call (CUB radix sort)
  const bool sorted = c.output_stage == 0 && c.n_beam >= kSortedBeams;
  int *skeys = nullptr, *sidx = nullptr;
  if (sorted) {
    const size_t n = size_t(c.n_beam);
    size_t temp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<const int*>(nullptr),
                                    static_cast<int*>(nullptr), static_cast<const int*>(nullptr),
                                    static_cast<int*>(nullptr), int(n), 0, 31, s);
    const size_t arr = (n * sizeof(int) + 255) / 256 * 256;
    const size_t need_sort = 4 * arr + temp;
    if (st->sort_bytes < need_sort) {
      if (stream_capturing(s))
        return fail(h, FTDX_ERR_CAPACITY, "image_beams: beam sort workspace needed while capturing");
      cudaStreamSynchronize(s);
      if (st->sort) cudaFree(st->sort);
      st->sort = nullptr;
      st->sort_bytes = 0;
      e = cudaMalloc(&st->sort, need_sort);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(h, FTDX_ERR_ALLOC, "image_beams: beam sort workspace of %zu bytes",
                    need_sort);
      }
      st->sort_bytes = need_sort;
    }
    char* base = static_cast<char*>(st->sort);
    int* keys_in = reinterpret_cast<int*>(base);
    int* idx_in = reinterpret_cast<int*>(base + arr);
    skeys = reinterpret_cast<int*>(base + 2 * arr);
    sidx = reinterpret_cast<int*>(base + 3 * arr);
    beam_keys_kernel<<<unsigned(std::min<int64_t>((int64_t(n) + 255) / 256, h->sm_count * 8)),
                       256, 0, s>>>(c.beam_pixels, c.n_beam, Ng, keys_in, idx_in);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cub::DeviceRadixSort::SortPairs(base + 4 * arr, temp, keys_in, skeys, idx_in, sidx,
                                          int(n), 0, 31, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "beam pixel sort");
  }
  for (int f0 = 0; f0 < c.n_chan; f0 += tile) {
    const int nf = std::min(tile, c.n_chan - f0);
    e = cudaMemsetAsync(st->grid, 0, size_t(nf) * size_t(plane) * sizeof(float2), s);
    if (e != cudaSuccess) return cuda_fail(h, e, "grid clear");
    {
      // a grid larger than the 64 MiB tile budget (one channel of Ng > 2896)
      // is scattered in row bands of at most 64 MiB per launch
      const int64_t tile_bytes = int64_t(nf) * plane * int64_t(sizeof(float2));
      const int bands = int(std::max<int64_t>(1, (tile_bytes + (int64_t(64) << 20) - 1) /
                                                     (int64_t(64) << 20)));
      const int rows = (Ng + bands - 1) / bands;
      const int64_t blocks = std::min<int64_t>((n_bl + 255) / 256, int64_t(h->sm_count) * 32);
      e = cudaSuccess;
      for (int r0 = 0; r0 < Ng && e == cudaSuccess; r0 += rows) {
        grid_scatter_kernel<<<unsigned(std::max<int64_t>(blocks, 1)), 256, 0, s>>>(
            static_cast<const float2*>(vis), reinterpret_cast<const float2*>(c.baseline_uv_m),
            c.freq_hz, c.taper, st->grid, n_bl, c.n_pol, Ng, f0, nf, c.cell_size_rad, r0,
            std::min(Ng, r0 + rows));
        e = cudaGetLastError();
      }
    }
    if (e != cudaSuccess) return cuda_fail(h, e, "grid scatter launch");
    if (c.output_stage == 1) {
      e = cudaMemcpyAsync(static_cast<float2*>(grid_out) + int64_t(f0) * plane, st->grid,
                          size_t(nf) * size_t(plane) * sizeof(float2), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return cuda_fail(h, e, "grid copy");
      continue;
    }
    const auto key = std::make_pair(Ng, nf);
    auto it = st->plans.find(key);
    if (it == st->plans.end()) {
      if (stream_capturing(s))
        return fail(h, FTDX_ERR_CAPACITY, "image_beams: FFT plan needed while capturing");
      cufftHandle plan = 0;
      int n[2] = {Ng, Ng};
      if (cufftPlanMany(&plan, 2, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, nf) !=
          CUFFT_SUCCESS)
        return fail(h, FTDX_ERR_CUDA, "image_beams: cufftPlanMany(%d x %d, %d) failed", Ng, Ng,
                    nf);
      it = st->plans.emplace(key, plan).first;
    }
    if (cufftSetStream(it->second, s) != CUFFT_SUCCESS ||
        cufftExecC2C(it->second, reinterpret_cast<cufftComplex*>(st->grid),
                     reinterpret_cast<cufftComplex*>(st->grid), CUFFT_INVERSE) != CUFFT_SUCCESS)
      return fail(h, FTDX_ERR_CUDA, "image_beams: inverse FFT failed");
    if (c.output_stage == 2) {
      e = cudaMemcpyAsync(static_cast<float2*>(grid_out) + int64_t(f0) * plane, st->grid,
                          size_t(nf) * size_t(plane) * sizeof(float2), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return cuda_fail(h, e, "image copy");
      continue;
    }
    if (sorted) {
      const int64_t total = int64_t(nf) * c.n_beam;
      beam_extract_sorted_kernel<<<unsigned(std::min<int64_t>((total + 255) / 256,
                                                               int64_t(h->sm_count) * 16)),
                                   256, 0, s>>>(st->grid, skeys, sidx,
                                                beams + int64_t(f0) * c.n_beam, plane, c.n_beam,
                                                nf, norm);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(h, e, "beam extraction launch");
    } else if (c.n_beam > 0) {
      const int total = nf * c.n_beam;
      beam_extract_kernel<<<unsigned(std::min((total + 255) / 256, h->sm_count * 8)), 256, 0, s>>>(
          st->grid, c.beam_pixels, beams + int64_t(f0) * c.n_beam, Ng, c.n_beam, nf, norm);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(h, e, "beam extraction launch");
    }
  }
  return FTDX_OK;
}
