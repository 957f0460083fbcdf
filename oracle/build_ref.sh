#!/usr/bin/env bash
# Builds oracle/_ref/libb40c_ref.so from the reference's own sources, where
# they lie in the read-only reference tree given as $1.
# Outputs go only to oracle/_ref/ (git-ignored).  Used to pin the C oracle and
# the host builders against the reference, and as the reference CPU baseline.
#
# The reference's serial CPU BFS (SimpleReferenceBfs) is defined inside its
# driver test/bfs/test_bfs.cu, whose other includes (GPU kernels using
# texture references) do not compile with CUDA 12, so the function's text is
# cut out of that file at build time into oracle/_ref/ and compiled by
# oracle/ref_harness.cpp together with the reference's builder headers.
set -euo pipefail
REF="${1:?usage: build_ref.sh <reference tree>}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
if [ ! -f "$REF/test/bfs/test_bfs.cu" ]; then
    echo "reference tree not found at $REF" >&2
    exit 2
fi
mkdir -p "$OUT"
# From the 'template<' line that opens SimpleReferenceBfs's declaration to the
# first closing brace in column 0 after the function name.
awk '
    /^template ?</ { buf = $0 "\n"; inbuf = 1; next }
    inbuf && !found { buf = buf $0 "\n"; if ($0 ~ /^void SimpleReferenceBfs\(/) { found = 1; printf "%s", buf; buf = "" } else if ($0 ~ /^[a-z].*\(/ && $0 !~ /^void SimpleReferenceBfs/) { inbuf = 0 } ; next }
    found && !done { print; if ($0 ~ /^}/) { done = 1 } }
' "$REF/test/bfs/test_bfs.cu" > "$OUT/simple_reference_bfs.inc"
if ! grep -q "SimpleReferenceBfs" "$OUT/simple_reference_bfs.inc"; then
    echo "could not extract SimpleReferenceBfs" >&2
    exit 3
fi
g++ -O2 -fPIC -shared -w \
    -I"$HERE" -I"$REF" -I"$REF/test" -I"$CUDA_HOME/include" \
    "$HERE/ref_harness.cpp" -o "$OUT/libb40c_ref.so.tmp" \
    -L"$CUDA_HOME/lib64" -lcudart_static -ldl -lpthread -lrt
mv "$OUT/libb40c_ref.so.tmp" "$OUT/libb40c_ref.so"
echo "built $OUT/libb40c_ref.so"
