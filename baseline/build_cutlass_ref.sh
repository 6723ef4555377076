#!/usr/bin/env bash
# Builds baseline/_ref/libref_cutlass_api.so: the reference's own public HERK
# API (cutlass_interface/cutlass_gemm_api.cu and gemm_blockscaled_dispatch.cu,
# with its CUTLASS tcgen05 sub-GEMM baseline and its direct kernels), compiled
# unmodified for sm_100a with nvcc 12.9 against the CUTLASS 4.5 headers that
# ship in this image, behind this directory's harness (cutlass_api_harness.cpp).
# The reference's CMake build refuses CUDA < 13 for Blackwell
# (cutlass_interface/CMakeLists.txt:97-103); the sources themselves compile.
# Definitions are the CMake defaults (cutlass_interface/CMakeLists.txt:196-430:
# 128 x 128 x 128 tiles, 1 x 1 clusters, FP6 and FP4 enabled) except the
# 64-row block-scaled tiles (COMPLEX_SM100_ENABLE_SMALL_M), which these
# CUTLASS headers reject.  Reads the reference tree ($FTD_REFERENCE, else a
# checkout named "reference" beside this repository) and the CUTLASS headers
# ($CUTLASS_DIR, else flashinfer's copy in site-packages); writes only into
# baseline/_ref/ (git-ignored).  About 15 minutes of compilation (the two
# units build in parallel).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${FTD_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
CI="$REF/cutlass_interface"
for f in "$CI/cutlass_gemm_api.cu" "$CI/gemm_blockscaled_dispatch.cu" "$CI/cutlass_gemm_api.h"; do
  [[ -f "$f" ]] || { echo "build_cutlass_ref: $f not found" >&2; exit 2; }
done
PY="${PYTHON:-python3}"
CUT="${CUTLASS_DIR:-$("$PY" -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')/flashinfer/data/cutlass}"
[[ -f "$CUT/include/cutlass/version.h" ]] || { echo "build_cutlass_ref: no CUTLASS at $CUT" >&2; exit 2; }
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
mkdir -p "$OUT"
DEFS=(-DCOMPLEX_FP8_SM100_MMA_M=128 -DCOMPLEX_FP8_SM100_MMA_N=128 -DCOMPLEX_FP8_SM100_MMA_K=128
      -DCOMPLEX_FP8_SM100_CLUSTER_M=1 -DCOMPLEX_FP8_SM100_CLUSTER_N=1
      -DCOMPLEX_SM100_BLKSCALED_MMA_M=128 -DCOMPLEX_SM100_BLKSCALED_MMA_N=128
      -DCOMPLEX_SM100_ENABLE_FP6=1 -DCOMPLEX_SM100_FP6_MMA_K=128
      -DCOMPLEX_SM100_ENABLE_FP4=1 -DCOMPLEX_SM100_FP4_MMA_K=256)
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 --expt-relaxed-constexpr
       --expt-extended-lambda -Xcompiler -fPIC "${DEFS[@]}"
       -I "$CUT/include" -I "$CUT/tools/util/include" -I "$CI" -I "$REF/include")
"$NVCC" "${FLAGS[@]}" -c "$CI/cutlass_gemm_api.cu" -o "$OUT/ref_cutlass_gemm_api.o" &
P1=$!
"$NVCC" "${FLAGS[@]}" -c "$CI/gemm_blockscaled_dispatch.cu" -o "$OUT/ref_blockscaled.o" &
P2=$!
wait $P1 || { kill $P2 2>/dev/null; wait $P2 2>/dev/null; echo "build_cutlass_ref: cutlass_gemm_api.cu failed" >&2; exit 1; }
wait $P2 || { echo "build_cutlass_ref: gemm_blockscaled_dispatch.cu failed" >&2; exit 1; }
"$NVCC" "${FLAGS[@]}" -x cu -c "$HERE/cutlass_api_harness.cpp" -o "$OUT/ref_cutlass_harness.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libref_cutlass_api.so.tmp" \
  "$OUT/ref_cutlass_harness.o" "$OUT/ref_cutlass_gemm_api.o" "$OUT/ref_blockscaled.o" -lcuda
mv "$OUT/libref_cutlass_api.so.tmp" "$OUT/libref_cutlass_api.so"
rm -f "$OUT/ref_cutlass_harness.o" "$OUT/ref_cutlass_gemm_api.o" "$OUT/ref_blockscaled.o"
echo "$OUT/libref_cutlass_api.so"
