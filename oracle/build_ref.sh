#!/usr/bin/env bash
# Builds the checkers under oracle/ (test infrastructure, never the product):
#   oracle/lib/liborules.so     the C restatement of the counting semantics
#   oracle/_ref/cpu01_harness   the reference's CPU_01_nonparallel sources,
#                               compiled where they lie, with ref_harness.cpp
# The second step runs only when the reference tree is present (REF_DIR,
# default: a `reference` checkout beside this repository); on a machine
# without it the prebuilt binary, if any, is kept.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_DIR="${REF_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
mkdir -p "$HERE/lib"
gcc -O2 -std=c11 -Wall -Wextra -shared -fPIC "$HERE/rules_oracle.c" -o "$HERE/lib/liborules.so"
SRC="$REF_DIR/CPU_01_nonparallel"
if [ -f "$SRC/SupportCounting.cpp" ]; then
  mkdir -p "$HERE/_ref"
  g++ -O3 -std=c++17 -pthread -I"$SRC" "$HERE/ref_harness.cpp" \
      "$SRC/FinalRule.cpp" "$SRC/RdfIndexes.cpp" "$SRC/RuleParser.cpp" "$SRC/SupportCounting.cpp" \
      -o "$HERE/_ref/cpu01_harness"
fi
