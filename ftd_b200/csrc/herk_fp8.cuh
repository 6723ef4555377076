// herk_fp8.cuh -- shared declarations of the correlator (HERK) kernels.
//
// Data layout in HBM (per channel c, N_c antennas, K_c time samples):
//   QC input   : [N_c][K_c] bytes, one complex sample per byte, high nibble =
//                Re, low nibble = Im, each sign-magnitude in [-7, 7]
//                (the reference's QC format, cutlass_interface/test_herk_int4.cu:41-45).
//   operand Z  : [2*N_c][zpitch] FP8 E4M3 bytes, zpitch = 2*Kp, Kp = K rounded
//                up to 64.  Row 2a is x_a = (re_t, im_t)_t and row 2a+1 is
//                y_a = (im_t, -re_t)_t, so that x_j . x_a = Re R_aj and
//                x_j . y_a = Im R_aj (the conjugate-permutation identity of
//                cutlass_interface/shared/herk_kernel_common.hpp:8-13).
//   output     : packed lower triangle, row-major, element (i, j <= i) at
//                i(i+1)/2 + j, interleaved (re, im) FP32 or FP16.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace ftdx {

constexpr int kBlockJ = 128;                 // UMMA M: column antennas j (x rows)
constexpr int kBlockI = 128;                 // row antennas i, two operand rows each
constexpr int kUmmaN = 2 * kBlockI;          // UMMA N = 256
constexpr int kKBytes = 128;                 // operand bytes of K per stage = 64 samples
constexpr int kSamplesPerStage = kKBytes / 2;
constexpr int kStages = 4;
constexpr int kABytes = kBlockJ * kKBytes;   // 16 KB
constexpr int kBBytes = kUmmaN * kKBytes;    // 32 KB
constexpr int kStageBytes = kABytes + kBBytes;
constexpr int kAccCols = kUmmaN;             // FP32 TMEM columns per accumulator
constexpr int kHerkThreads = 192;            // TMA warp, MMA warp, 4 epilogue warps
constexpr size_t kHerkSmem = 1024 + size_t(kStages) * kStageBytes + 256;

// One lower-triangle tile: channel, row block ti (i), column block tj (j), tj <= ti.
struct TileDesc {
  int32_t ch;
  uint16_t ti;
  uint16_t tj;
};

// Per-channel geometry.  row0 is the channel's first antenna row in the
// x-row view of Z (its Z rows start at 2*row0); out0 is the channel's first
// packed-triangle element in the output.
struct ChanDesc {
  int32_t n;
  int32_t kblocks;
  int64_t row0;
  int64_t out0;
  int64_t reserved;
};

struct HerkArgs {
  const TileDesc* tiles;
  const ChanDesc* chans;
  int32_t num_tiles;
  int32_t out_fp16;
  void* out;
  float alpha;
  float beta;
  uint32_t* status;
};

// Host-side launchers (herk_fp8.cu).
cudaError_t launch_qc_to_z(const uint8_t* qc, uint8_t* z, int64_t rows, int K, int Kp,
                           int sm_count, cudaStream_t s);
cudaError_t launch_fp16_to_z(const void* a16, uint8_t* z, int64_t rows, int K, int Kp,
                             int sm_count, cudaStream_t s);
cudaError_t launch_herk_fp8(const CUtensorMap& tmX, const CUtensorMap& tmZ, const HerkArgs& a,
                            int grid, cudaStream_t s);

}  // namespace ftdx
