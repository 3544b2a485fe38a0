#!/usr/bin/env bash
# Builds the reference engine's own file driver (landstats-us/postgis-cuda engine/harness.cu, unmodified) for
# sm_100a into oracle/_ref/harness. Test infrastructure: it runs on the GPU box to pin the CPU oracle and to time
# the reference engine on the same synthetic inputs. Needs the reference sources (read in place, not copied).
set -euo pipefail
REF=${REF:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$HERE/_ref"
if [ ! -f "$REF/engine/harness.cu" ]; then echo "reference sources not found at $REF" >&2; exit 1; fi
nvcc -std=c++17 -O3 -arch=sm_100a --expt-relaxed-constexpr -Xcompiler -fopenmp \
  -o "$HERE/_ref/harness" "$REF/engine/harness.cu" -lgomp
echo "built $HERE/_ref/harness"
