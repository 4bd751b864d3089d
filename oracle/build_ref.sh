#!/bin/bash
# ORACLE -- test infrastructure, not product code.
#
# Compiles the reference's own programs from their sources, where they lie in the reference
# tree, into oracle/_ref/ (git-ignored; it travels with the repository snapshot to the GPU
# box, which has no reference tree). Nothing is copied out of the reference.
#   scout_{mis,coloring,bfs,cc}   src/<p>/scout_<p>.cu with the reference's flags
#                                 (README.md:29-39), the arch pinned to sm_100a
#   greedy_color                  tools/greedy_color.cpp
#   ref_core_driver               oracle/ref_core_driver.cpp over core/*.h
# Set FORCE=1 to rebuild. The engines need nvcc and take a while; the rest is seconds.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# the reference tree: $SCOUT_REFERENCE_DIR, else `reference` beside the repository root
REF="${SCOUT_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
FORCE="${FORCE:-0}"
NVCC="${NVCC:-nvcc}"
CUDA_INC="$(dirname "$(command -v "$NVCC")")/../include"
[ -d "$REF" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
mkdir -p "$OUT"

need() { [ "$FORCE" = "1" ] || [ ! -x "$1" ] || [ "$2" -nt "$1" ]; }

if need "$OUT/greedy_color" "$REF/tools/greedy_color.cpp"; then
    g++ -O3 "$REF/tools/greedy_color.cpp" -o "$OUT/greedy_color"
fi
if need "$OUT/ref_core_driver" "$HERE/ref_core_driver.cpp"; then
    g++ -O2 -std=c++17 -I"$REF/core" -I"$CUDA_INC" "$HERE/ref_core_driver.cpp" -o "$OUT/ref_core_driver"
fi
if [ "${SCOUT_REF_ENGINES:-1}" = "1" ]; then
    for p in mis coloring bfs cc; do
        if need "$OUT/scout_$p" "$REF/src/$p/scout_$p.cu"; then
            "$NVCC" -O3 -std=c++17 -Xcompiler -fopenmp -gencode arch=compute_100a,code=sm_100a \
                -I"$REF" "$REF/src/$p/scout_$p.cu" -o "$OUT/scout_$p" &
        fi
    done
    wait
fi
echo "reference programs in $OUT"
