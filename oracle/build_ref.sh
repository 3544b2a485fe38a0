#!/usr/bin/env bash
# Builds the reference engine's own file driver (landstats-us/postgis-cuda engine/harness.cu, unmodified) for
# sm_100a into oracle/_ref/harness. Test infrastructure: it runs on the GPU box to pin the CPU oracle, as the
# pair-level checker at the benchmarked sizes, and as the timed reference arm. Needs the reference sources, read in
# place (not copied):   oracle/build_ref.sh <reference source tree>
set -euo pipefail
if [ $# -ne 1 ]; then echo "usage: $0 <reference source tree>" >&2; exit 2; fi
REF="$1"
HERE="$(cd "$(dirname "$0")" && pwd)"
if [ ! -f "$REF/engine/harness.cu" ]; then echo "reference sources not found at $REF" >&2; exit 1; fi
mkdir -p "$HERE/_ref"
nvcc -std=c++17 -O3 -arch=sm_100a --expt-relaxed-constexpr -Xcompiler -fopenmp \
  -o "$HERE/_ref/harness" "$REF/engine/harness.cu" -lgomp
echo "built $HERE/_ref/harness"
