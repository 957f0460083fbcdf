#!/usr/bin/env bash
# Builds oracle/_ref/test_bfs_dropin: the reference's own BFS driver
# (test/bfs/test_bfs.cu, RunTests and main), compiled unchanged from where it
# lies in the read-only reference tree against this repository's drop-in
# headers (include/b40c/...) and linked to back40computing_b200/lib/libb40c_bfs.so.
# The include path puts include/ first; only the driver's own test helpers
# (test/b40c_test_util.h and the b40c/util/random_bits.cuh it includes) come
# from the reference tree.  Output goes only to oracle/_ref/ (git-ignored).
#
#   oracle/build_dropin.sh <reference tree>
set -euo pipefail
REF="${1:?usage: build_dropin.sh <reference tree>}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT="$(dirname "$HERE")"
OUT="$HERE/_ref"
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
LIB="$ROOT/back40computing_b200/lib"
if [ ! -f "$REF/test/bfs/test_bfs.cu" ]; then
    echo "reference driver not found under $REF" >&2
    exit 2
fi
if [ ! -f "$LIB/libb40c_bfs.so" ]; then
    echo "build the library first (python -m back40computing_b200.build)" >&2
    exit 2
fi
mkdir -p "$OUT"
"$CUDA_HOME/bin/nvcc" -std=c++17 -O2 -w -gencode arch=compute_100a,code=sm_100a \
    -I"$ROOT/include" -I"$REF/test" -Xcompiler -idirafter,"$REF" \
    "$REF/test/bfs/test_bfs.cu" -o "$OUT/test_bfs_dropin.tmp" \
    -L"$LIB" -lb40c_bfs -Xlinker -rpath -Xlinker '$ORIGIN/../../back40computing_b200/lib'
mv "$OUT/test_bfs_dropin.tmp" "$OUT/test_bfs_dropin"
echo "built $OUT/test_bfs_dropin"
