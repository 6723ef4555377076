#!/usr/bin/env bash
# Builds oracle/_ref/libref_herk.so from the reference's own host correlator
# code.  Reads the reference tree ($FTD_REFERENCE, else a checkout named
# "reference" beside this repository) and writes only into oracle/_ref/
# (git-ignored).  The extracted text is never committed; ref_harness.cpp
# (ours) includes it.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${FTD_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
T1="$REF/cutlass_interface/test_herk_int4.cu"
T2="$REF/tests/visibility_pipeline_test.cpp"
if [[ ! -f "$T1" || ! -f "$T2" ]]; then
  echo "build_ref: reference sources not found under $REF" >&2
  exit 2
fi
mkdir -p "$OUT"
# Print the definition of a static function: from its signature line to the
# first line that is a lone closing brace.
extract() {  # file name
  awk -v name="$2" '
    !on && $0 ~ "^static .*[ *&]" name "\\(" { on = 1 }
    on { print }
    on && $0 ~ /^}[ \t]*$/ { exit }
  ' "$1"
}
{
  echo "// extracted from the reference tree by oracle/build_ref.sh -- do not commit"
  extract "$T1" encode_int4
  extract "$T1" cpu_herk
  extract "$T2" decode_qc_byte
  extract "$T2" cpu_herk_batch_first
  extract "$T2" cpu_herk_ftd
} > "$OUT/ref_extract.inc"
for f in encode_int4 cpu_herk decode_qc_byte cpu_herk_batch_first cpu_herk_ftd; do
  grep -q "$f(" "$OUT/ref_extract.inc" || { echo "build_ref: $f not found" >&2; exit 3; }
done
# The XEngine and imaging helpers: device functors and functions of the
# reference's kernels (compiled host-side by ref_harness.cpp with stand-ins
# for the CUDA qualifiers) and the XEngine test's own host decode.
span() {  # file start-regex end-regex: from the first line matching start
  awk -v a="$2" -v b="$3" '
    !on && $0 ~ a { on = 1; print; next }
    on { print }
    on && $0 ~ b { exit }
  ' "$1"
}
K1="$REF/include/kernels/promote_data.cuh"
K2="$REF/include/kernels/tri_from_herm.cuh"
K3="$REF/include/kernels/imaging_kernels.cuh"
T3="$REF/tests/xengine_test.cpp"
for f in "$K1" "$K2" "$K3" "$T3"; do
  [[ -f "$f" ]] || { echo "build_ref: $f not found" >&2; exit 2; }
done
{
  echo "// extracted from the reference tree by oracle/build_ref.sh -- do not commit"
  span "$K1" "template <typename Arg> struct DataPromote [{]" "^  [}];"
  span "$K2" "template <typename Arg> struct HermToTri [{]" "^  [}];"
  grep -m1 "static constexpr double C_LIGHT" "$K3"
  span "$K3" "void tri_decode[(]" "^[}]"
  span "$K3" "void uv_cell[(]" "^[}]"
  span "$T3" "void promote_to_float[(]" "^[}]"
} > "$OUT/ref_extract_kernels.inc"
for f in "struct DataPromote" "struct HermToTri" "C_LIGHT" "tri_decode(" "uv_cell(" "promote_to_float("; do
  grep -q "$f" "$OUT/ref_extract_kernels.inc" || { echo "build_ref: $f not found" >&2; exit 3; }
done
/usr/bin/g++ -O3 -fopenmp -march=x86-64-v3 -std=c++17 -fPIC -shared -I"$OUT" \
    "$HERE/ref_harness.cpp" -o "$OUT/libref_herk.so.tmp"
mv "$OUT/libref_herk.so.tmp" "$OUT/libref_herk.so"
echo "$OUT/libref_herk.so"
