#!/usr/bin/env bash
# Builds baseline/_ref/libref_direct_herk.so: the reference's own Blackwell
# direct HERK kernel (herk_direct_fp8_precast_kernel and its launcher,
# cutlass_interface/shared/herk_kernel_common.hpp:1-461, plain CUDA with
# mma.sync and cp.async) and its INT4 -> interleaved FP8 cast
# (qc_to_fp8_lut_256 and cast_int4_to_fp8_interleaved,
# cutlass_interface/cutlass_gemm_api.cu:1436-1623), compiled for sm_100a with
# nvcc behind this directory's harness (direct_herk_harness.cu).  The
# reference's CMake build needs CUDA >= 13 (cutlass_interface/CMakeLists.txt:
# 97-103); these sources need only cutlass::Status, FillMode and CUDA_CHECK,
# for which the harness gives stand-ins.  Reads the reference tree
# ($FTD_REFERENCE, else a checkout named "reference" beside this
# repository) and writes only into baseline/_ref/ (git-ignored); the
# extracted text is never committed.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${FTD_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
H1="$REF/cutlass_interface/shared/herk_kernel_common.hpp"
C1="$REF/cutlass_interface/cutlass_gemm_api.cu"
for f in "$H1" "$C1"; do
  [[ -f "$f" ]] || { echo "build_direct_ref: $f not found" >&2; exit 2; }
done
mkdir -p "$OUT"
# the direct kernel section: from the top of the header to the small-K helpers
awk '/^\/\/ Direct load helper: vectorized global/ { exit } { print }' "$H1" \
  | sed '$d' > "$OUT/ref_direct_herk.inc"
# the INT4 -> FP8 LUT and cast: from the LUT's comment to the FP16 section
awk '/^\/\/\/ @brief 256-entry byte->FP8-pair LUT/ { on = 1 }
     /^\/\/ ---- INT4 -> FP16 planar/ { exit }
     on { print }' "$C1" > "$OUT/ref_qc_cast.inc"
grep -q "herk_direct_fp8_precast_kernel" "$OUT/ref_direct_herk.inc"
grep -q "launch_herk_direct_fp8_precast" "$OUT/ref_direct_herk.inc"
grep -q "cast_int4_to_fp8_interleaved_kernel" "$OUT/ref_qc_cast.inc"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Xcompiler -fPIC -shared \
  -I"$OUT" "$HERE/direct_herk_harness.cu" -o "$OUT/libref_direct_herk.so.tmp"
mv "$OUT/libref_direct_herk.so.tmp" "$OUT/libref_direct_herk.so"
echo "$OUT/libref_direct_herk.so"
