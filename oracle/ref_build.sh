#!/usr/bin/env bash
# Build the reference's own kernels (frsykzk/MPS_CUDA) for sm_100a, driven by ref_harness.cu.
# Test infrastructure: outputs go only to oracle/_ref/ (git-ignored). The reference sources
# are read where they lie; the build copies in oracle/_ref/src_* are transcoded from
# Shift-JIS (CP932) to UTF-8, which nvcc needs, and patched as follows:
#   * kernel.cu:849  `treal3 synvec;` is initialised to zero (it is summed into while
#                    uninitialised);
#   * FP64 variant:  const.cuh:52-53 typedef switched to double and the f-suffixed float
#                    literals of const.cuh / kernel.cu promoted to double literals;
#   * corrected-gradient variants (libref_mps_corr_*): the `#if 0` in front of the
#                    corrected-matrix d_PrsGrdTrm (kernel.cu:1434) switched to `#if 1`, so
#                    that the reference's own alternative kernel is compiled instead of the
#                    default one (kernel.cu:1650-1795).
# main.cu is not built: ref_harness.cu takes its place. The reference has no build files,
# so this script is the whole recipe.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
# the reference checkout: MPS_REFERENCE_DIR, else a directory named `reference` beside
# this repository
REF="${MPS_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-nvcc}"
if [ ! -f "$REF/kernel.cu" ]; then
    echo "reference sources not found in $REF" >&2
    exit 3
fi
mkdir -p "$OUT/src_f32" "$OUT/src_f64"
for f in class.cuh const.cuh kernel.cu; do
    iconv -f CP932 -t UTF-8 "$REF/$f" > "$OUT/src_f32/$f"
done
sed -i 's/^\(\s*\)treal3 synvec;/\1treal3 synvec = { 0.0f, 0.0f, 0.0f };/' "$OUT/src_f32/kernel.cu"
grep -q 'treal3 synvec = { 0.0f' "$OUT/src_f32/kernel.cu"
cp "$OUT/src_f32/"* "$OUT/src_f64/"
sed -i 's/^typedef float real;/typedef double real;/' "$OUT/src_f64/const.cuh"
grep -q '^typedef double real;' "$OUT/src_f64/const.cuh"
sed -i -E 's/([0-9]+\.[0-9]*)f([^0-9A-Za-z_]|$)/\1\2/g' "$OUT/src_f64/const.cuh" "$OUT/src_f64/kernel.cu"

for v in f32 f64; do
    mkdir -p "$OUT/src_corr_$v"
    cp "$OUT/src_$v/"* "$OUT/src_corr_$v/"
    sed -i '/^#if 0\r\?$/{N;s/^#if 0\(\r\?\n__global__ void d_PrsGrdTrm(\)/#if 1\1/}' "$OUT/src_corr_$v/kernel.cu"
    grep -A1 '^#if 1' "$OUT/src_corr_$v/kernel.cu" | grep -q '__global__ void d_PrsGrdTrm('
done

FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -shared -Xcompiler -fPIC
       -Xcompiler -w -include "$HERE/ref_compat.h")
for v in f32 f64 corr_f32 corr_f64; do
    "$NVCC" "${FLAGS[@]}" -I"$OUT/src_$v" -o "$OUT/libref_mps_$v.so" \
        "$HERE/ref_harness.cu" "$OUT/src_$v/kernel.cu"
done
echo "built $OUT/libref_mps_{f32,f64,corr_f32,corr_f64}.so"
