#!/usr/bin/env bash
# Builds the reference's own GPU library (GPU_03: gpu_rules_lib.cu with its
# RdfIndexes / RuleParser / FinalRule sources, compiled where they lie) for
# sm_100a into baseline/_ref/gpu03/libgpu_rules.so, as the per-rule GPU
# comparator of bench.py --gpu03.  Nothing of the reference is copied into
# this repository; the output directory is git-ignored.  Runs only where the
# reference tree is present (REF_DIR, default: a `reference` checkout
# beside this repository).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_DIR="${REF_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
SRC="$REF_DIR/GPU_03"
if [ ! -f "$SRC/gpu_rules_lib.cu" ]; then
  echo "reference GPU_03 sources not found under $REF_DIR; keeping any prebuilt library" >&2
  exit 0
fi
OUT="$HERE/_ref/gpu03"
mkdir -p "$OUT"
nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -shared -Xcompiler -fPIC -I"$SRC" \
     "$SRC/gpu_rules_lib.cu" "$SRC/RdfIndexes.cpp" "$SRC/RuleParser.cpp" "$SRC/FinalRule.cpp" \
     -o "$OUT/libgpu_rules.so"
echo "built $OUT/libgpu_rules.so"
