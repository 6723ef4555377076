// herk_fp8.cuh -- shared declarations of the correlator (HERK) kernels.
//
// Data layout in HBM (per channel c, N_c inputs, K_c time samples):
//   QC input   : [N_c][K_c] bytes, one complex sample per byte, high nibble =
//                Re, low nibble = Im, each sign-magnitude in [-7, 7]
//                (the reference's QC format, cutlass_interface/test_herk_int4.cu:41-45).
//   operand Z  : two FP8 E4M3 planes, Z[p][row][Kp], p = 0 holds Re, p = 1
//                holds Im, Kp = K rounded up to 128 and zero-padded.  Rows of
//                all channels are stacked (channel c starts at row0_c).
//   output     : packed lower triangle, row-major, element (i, j <= i) at
//                i(i+1)/2 + j, interleaved (re, im) FP32 or FP16.
//
// Complex arithmetic on real tensor-core products (per k-step, column
// antennas j in the MMA's M dimension, row antennas i in its N dimension):
//   Re R_ij += Re_j . Re_i + Im_j . Im_i
//   Im R_ij += Re_j . Im_i - Im_j . Re_i      (negate-A bit of the MMA)
// which is exactly 8 real FLOPs per complex multiply-accumulate.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

namespace ftdx {

constexpr int kTile = 128;                   // antennas per operand tile (M = N = 128)
constexpr int kStageK = 128;                 // samples per pipeline stage (= bytes per plane row)
constexpr int kPlaneBytes = kTile * kStageK; // 16 KB
constexpr int kStageBytes = 4 * kPlaneBytes; // A_re, A_im, B_re, B_im
constexpr int kStages = 3;
constexpr int kAccCols = 2 * kTile;          // FP32 TMEM columns per accumulator: Re | Im
constexpr int kEpiWarps = 8;                 // two per TMEM lane quarter
constexpr int kHerkThreads = 64 + 32 * kEpiWarps;  // TMA warp, MMA warp, epilogue warps
// Epilogue staging for bulk stores: per half of the epilogue warps, two
// buffers of kStgRows triangle-row segments (128 complex64 = 1 KB each, plus
// 16 B so a row can keep the 16-byte phase of its global address).
constexpr int kStgRows = 8;
constexpr int kStgRowBytes = kTile * 8 + 16;
constexpr int kStgBytes = 2 /*halves*/ * 2 /*buffers*/ * kStgRows * kStgRowBytes;
constexpr size_t kHerkSmem = 1024 + size_t(kStages) * kStageBytes + kStgBytes + 256;
static_assert(((kTile / 2) / kStgRows) % 2 == 0, "bulk tiles end on staging buffer 1");
// Fused promotion (store-mode flag kStoreFused, QC input): the producer loads
// raw QC bytes by TMA and kConvWarps converter warps write the E4M3 operand
// planes into shared memory, so no operand planes exist in HBM.  Two operand
// stages and three raw stages (128 A rows + 128 B rows of 128 QC bytes); no
// bulk-store staging.
constexpr int kConvWarps = 4;
constexpr int kConvThreads = 32 * kConvWarps;
constexpr int kFusedThreads = kHerkThreads + kConvThreads;
constexpr int kFusedStages = 2;
constexpr int kRawStages = 3;
constexpr int kRawStageBytes = 2 * kPlaneBytes;
constexpr size_t kFusedSmem =
    1024 + size_t(kFusedStages) * kStageBytes + size_t(kRawStages) * kRawStageBytes + 256;
static_assert(kFusedSmem <= 232448, "shared memory per CTA");

// One lower-triangle tile: channel, row block ti (i), column block tj (j), tj <= ti.
struct TileDesc {
  int32_t ch;
  uint16_t ti;
  uint16_t tj;
};

// Per-channel geometry.  row0 is the channel's first row in each plane of Z;
// the channel's packed triangle starts at out_ptr when it is non-zero (a
// device address), else at element out0 of HerkArgs::out.
struct ChanDesc {
  int32_t n;
  int32_t kblocks;
  int64_t row0;
  int64_t out0;
  int64_t out_ptr;
  int32_t kb0;  // first k-block (split-K: each split is its own channel entry)
  int32_t pad;
};

// One channel of a batched call with its own input geometry: the promotion
// pass gathers rows active[0..n) (or rows 0..n) of a [rows][lda] QC block.
struct GatherDesc {
  const uint8_t* a;
  const int32_t* active;  // nullptr: all rows
  int64_t lda;
  int64_t row0;           // first row in each plane of Z
  int32_t n;
  int32_t k;
};

struct HerkArgs {
  const TileDesc* tiles;
  const ChanDesc* chans;
  int32_t num_tiles;
  int32_t out_fp16;
  int32_t bulk_store;  // 1: interior tiles leave through shared memory + bulk copies
  // 0: packed lower triangle (element (i, j <= i) at i(i+1)/2 + j);
  // 1: packed upper triangle, row-major (element (r, c >= r) at
  //    r*n - r(r-1)/2 + c - r, holding sum_t conj(v_r) v_c: the XEngine's
  //    triangular format); 2: full n x n matrix of sum_t conj(v_r) v_c (the
  //    XEngine's Hermitian format).  Formats 1 and 2: single-CTA kernel,
  //    direct stores, beta = 0, no Kahan.
  int32_t out_format;
  void* out;
  float alpha;
  float beta;
  uint32_t* status;
  // K segments: segment s pairs the A (j) operand's k-blocks seg_a[s] + kk
  // with the B (i) operand's k-blocks seg_b[s] + kk, kk < kblocks, all
  // accumulated into one result (nseg = 1, offsets 0: a plain HERK).
  int32_t nseg;
  int32_t seg_a[3];
  int32_t seg_b[3];
  int32_t kahan;            // 1: Kahan-accumulate into out (sum) and out2 (compensation)
  const float* chan_scale;  // per-channel result multiplier (nullptr: 1)
  void* out2;
  // 1: Z holds packed FP6 E3M2 planes (TMA 16 x U6 type): the MMAs read E3M2
  // operands and each load delivers 3/4 of the FP8 bytes
  int32_t fp6;
  // 1: Z holds signed 8-bit planes (QC values exact); CTA-pair kernel only:
  // kind::i8 MMAs into S32 accumulators, converted to FP32 by the epilogue
  int32_t s8;
};

// A persistent CTA's walk over its tiles (first, first + step, ...) with the
// descriptors loaded ahead: the tile descriptor two tiles ahead and the
// channel descriptor one tile ahead (its index comes from a tile descriptor
// that arrived a tile earlier), so that no role waits on global memory at a
// tile boundary.  Loads past the end of the list are not issued.
struct TileWalk {
  const TileDesc* tiles;
  const ChanDesc* chans;
  int t, step, num;
  TileDesc td, td1, td2;  // this tile, the next, the one after
  ChanDesc cd, cd1;       // this tile's channel, the next tile's
  __device__ __forceinline__ TileWalk(const TileDesc* tiles_, const ChanDesc* chans_, int num_,
                                      int first, int step_)
      : tiles(tiles_), chans(chans_), t(first), step(step_), num(num_) {
    td = tile_at(t);
    cd = chan_of(td, t);
    td1 = tile_at(t + step);
    cd1 = chan_of(td1, t + step);
    td2 = tile_at(t + 2 * step);
  }
  __device__ __forceinline__ TileDesc tile_at(int u) const {
    return u < num ? tiles[u] : TileDesc{0, 0, 0};
  }
  __device__ __forceinline__ ChanDesc chan_of(const TileDesc& d, int u) const {
    return u < num ? chans[d.ch] : ChanDesc{};
  }
  __device__ __forceinline__ bool valid() const { return t < num; }
  __device__ __forceinline__ void advance() {
    t += step;
    td = td1;
    cd = cd1;
    td1 = td2;
    cd1 = chan_of(td1, t + step);
    td2 = tile_at(t + 2 * step);
  }
};

// A plain single-segment argument block.
inline HerkArgs herk_args_default() {
  HerkArgs a{};
  a.nseg = 1;
  a.alpha = 1.f;
  return a;
}

// Raises `kernel`'s dynamic shared-memory limit to `bytes` on the current
// device, once per (device, kernel): CUDA keeps this attribute per device, so
// a process driving several GPUs sets it on each.  Thread-safe (ftdx_api.cu).
cudaError_t ensure_smem_limit(const void* kernel, size_t bytes);
// Records the text of a failure of an entry point that takes no handle, for
// the calling thread; ftdx_last_error(NULL) returns it (ftdx_api.cu).
void set_thread_error(const char* fmt, ...);

// Host-side launchers (herk_fp8.cu).
// neg_plane: also write plane 2 = -Re (CTA-pair kernel operand)
cudaError_t launch_qc_to_planes(const uint8_t* qc, uint8_t* z, int64_t rows, int K, int Kp,
                                cudaStream_t s, bool neg_plane = false);
// Signed 8-bit planes (same layout as the E4M3 planes) for the s8 operand form.
cudaError_t launch_qc_to_planes_s8(const uint8_t* qc, uint8_t* z, int64_t rows, int K, int Kp,
                                   cudaStream_t s, bool neg_plane = false);
// Packed FP6 E3M2 planes (row pitch 3 Kp / 4 bytes) for the fp6 operand form.
cudaError_t launch_qc_to_planes6(const uint8_t* qc, uint8_t* z, int64_t rows, int K, int Kp,
                                 cudaStream_t s, bool neg_plane = false);
// Raw packet-ordered QC input (corner_turn.cu): geometry of the promotion.
struct FtdGeom {
  int n_ant, n_chan, n_pol, n_ti;  // antennas, channels, polarisations, time_inner
  int K;                           // samples per (chan, pol, ti) and antenna
  int n_time;                      // K * n_ti
  int pol_sum;                     // rows hold all pols back to back (n_pol*K columns)
  int Kp;                          // padded row length (multiple of kStageK)
  int64_t rows;                    // plane rows = n_ant * batches
  int neg_plane;                   // also write plane 2 = -Re
  // layout 0 source offset of (sample k, block z, slice byte s) =
  //   k*t_stride + z*z_stride + s  (0, 0: the [t][ant][chan][pol] strides)
  int64_t t_stride, z_stride;
  int twos;                        // (4,4)b two's complement bytes, low nibble Re
};
// layout 0: [t][ant][chan][pol], t = k*n_ti + ti; 1: [chan][pol][ant][t], t = ti*K + k.
cudaError_t launch_ftd_to_planes(const uint8_t* raw, uint8_t* z, const FtdGeom& g, int layout,
                                 int sm_count, cudaStream_t s);
// Plane 2 = -(plane 0), planes of plane_bytes each (a multiple of 16).
cudaError_t launch_negate_plane(uint8_t* z, int64_t plane_bytes, int sm_count, cudaStream_t s);
cudaError_t launch_fp16_to_planes(const void* a16, uint8_t* z, int64_t rows, int K, int Kp,
                                  cudaStream_t s);
// Gathered promotion for `nch` channels with a common plane pitch Kp
// (>= every channel's K rounded up to 128); each channel's rows are
// zero-padded from its K up to its own K rounded up to 128.  neg_plane: also
// write plane 2 = -Re (CTA-pair kernel operand).
cudaError_t launch_gather_qc_to_planes(const GatherDesc* g, int nch, int max_n, uint8_t* z,
                                       int64_t total_rows, int Kp, cudaStream_t s,
                                       int neg_plane = 0);
cudaError_t launch_herk_fp8(const CUtensorMap& tmZ, const HerkArgs& a, int grid, cudaStream_t s);
// The single-CTA kernel with fused promotion: tmQ maps the raw QC bytes
// [rows][K] (2-D, 128 x 128-byte boxes, no swizzle); a.nseg must be 1,
// a.out_format 0 and a.bulk_store 0.
cudaError_t launch_herk_fp8_fused(const CUtensorMap& tmQ, const HerkArgs& a, int grid,
                                  cudaStream_t s);
// Split-K reduction: C[c] = alpha * cs_c * sum_s ws[c*splits + s] + beta * C[c].
cudaError_t launch_split_reduce(const float2* ws, void* out, int out_fp16, int64_t P, int batch,
                                int splits, float alpha, float beta, const float* chan_scale,
                                int sm_count, cudaStream_t s);
// CTA-pair variant: tiles of 256 column x 128 row inputs (TileDesc::tj counts
// 256-input blocks); tmZ covers three planes (Re, Im, -Re), boxes of 128
// rows; grid even.
cudaError_t launch_herk_fp8_pair(const CUtensorMap& tmZ, const HerkArgs& a, int grid,
                                 cudaStream_t s);
// Number of 2-CTA clusters of the pair kernel that fit on the device at once.
cudaError_t herk_fp8_pair_max_clusters(int sm_count, int* clusters);
// Gain-calibration loss and gradient over packed triangles (gain_grad.cu).
cudaError_t launch_gain_grad(const float2* robs, const float2* rmod, const float* w,
                             const float2* g, int n, int nchan, double* grad, double* loss,
                             cudaStream_t s);
// Adjoint dV = (G + G^H) V (adjoint.cu); n must be a multiple of 8.
size_t adjoint_workspace_bytes(int n, int K, int batch);
cudaError_t launch_adjoint(const void* G, const uint8_t* V, void* dV, int n, int K, int batch,
                           uint8_t* ws, int sm_count, uint32_t* status, void* encode_fn,
                           cudaStream_t s);
// Per-channel max |Re|, |Im| of float complex input (bits of a float; caller zeroes).
cudaError_t launch_channel_amax(const void* a, int64_t per_chan, int batch, uint32_t* amax_bits,
                                int sm_count, cudaStream_t s);
// NVFP4 correlator for float complex input (herk_fp4.cu).  Tiles: ti over 64
// row inputs, tj over 128 column inputs; kblocks = nvfp4_kblocks(K).
// phases: 1 = the quantiser passes (they also write each channel's lo extent
// into chans[c].pad), 2 = the correlator, 3 = both.
// pair: the CTA-pair kernel (tiles from nvfp4_pair_tiles: tj over 256 column
// inputs, ti over 112 row inputs), when nvfp4_pair_limit() >= 1.
size_t nvfp4_workspace_bytes(int n, int batch, int K, int split = 0, int pair = 0);
int nvfp4_kblocks(int K);
int nvfp4_pair_limit();
void nvfp4_pair_tiles(int n, int ch, std::vector<TileDesc>& out);
cudaError_t launch_nvfp4(const void* A, int64_t rows, int K, int n, int batch, uint8_t* ws,
                         const TileDesc* tiles, const ChanDesc* chans, int num_tiles, void* C,
                         float alpha, float beta, uint32_t* status, int sm_count, void* encode_fn,
                         cudaStream_t s, int split = 0, int pair = 0, int phases = 3);
// Float complex [rows][K] -> scaled E4M3 planes of pitch zpitch (precision.cu);
// neg: also plane 2 (-Re).  arrive: 32 words per channel, 128-byte aligned,
// directly followed by amax_bits[batch] (the one-pass cooperative kernel
// needs that placement; any other takes the three-kernel path).
cudaError_t launch_float_to_planes(const void* a, uint8_t* z, int64_t rows, int K, int Kp,
                                   int zpitch, int n, int batch, int split, int neg,
                                   float* qscale, float* out_scale, uint32_t* amax_bits,
                                   uint32_t* arrive, uint32_t* status, int sm_count,
                                   cudaStream_t s);

}  // namespace ftdx
