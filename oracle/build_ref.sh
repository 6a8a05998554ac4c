#!/usr/bin/env bash
# Builds the reference XTNeighbor-streaming from its own sources (read in place, never
# copied) into oracle/_ref/, for use as a checker and as the benchmark's reference arm only:
#   _ref/xt_neighbor_ref - the reference CLI (S/src/cli.cu, one translation unit), sm_100a
#   _ref/ref_perform     - the reference's xtn_perform timed as a library call (ref_perform.cu)
#   _ref/ref_harness     - host harness around the reference's variant generator and codec
# Usage: oracle/build_ref.sh [reference_root]
# The reference checkout is taken from the argument, else from $XTN_REFERENCE_ROOT, else from
# a directory named "reference" beside this repository.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF=${1:-${XTN_REFERENCE_ROOT:-$(dirname "$(dirname "$HERE")")/reference}}
SRC="$REF/xtneighbor_streaming/src"
OUT="$HERE/_ref"
if [ ! -f "$SRC/cli.cu" ]; then
    echo "build_ref: reference sources not found under $SRC; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ ! -x "$OUT/ref_harness" ] || [ "$HERE/ref_harness.cu" -nt "$OUT/ref_harness" ]; then
    "$NVCC" -O2 -w -gencode arch=compute_100a,code=sm_100a -I "$SRC" -o "$OUT/ref_harness" "$HERE/ref_harness.cu"
fi
if [ ! -x "$OUT/xt_neighbor_ref" ]; then
    "$NVCC" -O3 -w -gencode arch=compute_100a,code=sm_100a -o "$OUT/xt_neighbor_ref" "$SRC/cli.cu"
fi
if [ ! -x "$OUT/ref_perform" ] || [ "$HERE/ref_perform.cu" -nt "$OUT/ref_perform" ]; then
    "$NVCC" -O3 -w -gencode arch=compute_100a,code=sm_100a -I "$SRC" -o "$OUT/ref_perform" "$HERE/ref_perform.cu"
fi
echo "build_ref: ok ($OUT)"
