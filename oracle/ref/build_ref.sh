#!/usr/bin/env bash
# Compiles the reference warpcore headers (read in place from the reference
# checkout) into golden-vector and timing programs under oracle/_ref/.
# Needs the reference sources, so it runs in the build container only; the
# binaries it writes travel with the repository snapshot.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ORACLE="$(dirname "$HERE")"
REF="${WC_REFERENCE_DIR:-/root/reference}"
OUT="$ORACLE/_ref"
if [ ! -d "$REF/include/warpcore" ]; then
    echo "reference sources not found at $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT/include/helpers"
cp "$HERE/cuda_helpers_standin.cuh" "$OUT/include/helpers/cuda_helpers.cuh"
cp "$HERE/packed_types_standin.cuh" "$OUT/include/helpers/packed_types.cuh"
NVCC="${NVCC:-nvcc}"
FLAGS=(-std=c++17 --expt-extended-lambda --expt-relaxed-constexpr -O3
       -gencode arch=compute_100a,code=sm_100a -lineinfo
       -I"$REF/include" -I"$OUT/include" -I"$ORACLE" -w)
gcc -O2 -std=c11 -fPIC -pthread -c "$ORACLE/wc_oracle.c" -o "$OUT/wc_oracle.o"
"$NVCC" "${FLAGS[@]}" "$HERE/make_golden.cu" "$OUT/wc_oracle.o" -o "$OUT/make_golden" -lm
if [ -f "$HERE/ref_bench.cu" ]; then
    "$NVCC" "${FLAGS[@]}" "$HERE/ref_bench.cu" "$OUT/wc_oracle.o" -o "$OUT/ref_bench" -lm
fi
echo "built reference programs in $OUT"
