#!/usr/bin/env bash
# Builds the reference warpcore (read in place from the reference checkout)
# for sm_100a into baseline/_ref/libwarpcore_ref_bench.so, the GPU baseline
# that bench.py times next to this library.  Needs the reference sources, so
# it runs in the build container; the library travels with the snapshot.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT="$(dirname "$HERE")"
REF="${WC_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/include/warpcore" ]; then
    echo "reference sources not found at $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT/include/helpers"
cp "$ROOT/oracle/ref/cuda_helpers_standin.cuh" "$OUT/include/helpers/cuda_helpers.cuh"
cp "$ROOT/oracle/ref/packed_types_standin.cuh" "$OUT/include/helpers/packed_types.cuh"
"${NVCC:-nvcc}" -std=c++17 --expt-extended-lambda --expt-relaxed-constexpr -O3 \
    -gencode arch=compute_100a,code=sm_100a -lineinfo -w \
    -I"$REF/include" -I"$OUT/include" -Xcompiler -fPIC -shared \
    "$HERE/ref_gpu_bench.cu" -o "$OUT/libwarpcore_ref_bench.so"
echo "built $OUT/libwarpcore_ref_bench.so (MAXBLOCKSIZE=1024)"
