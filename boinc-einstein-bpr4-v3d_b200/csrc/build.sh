#!/bin/sh
# Builds libbrp_cuda.so (the package's CUDA backend) for sm_100a.
# Usage: build.sh [output path]   (default: the package root)
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=${1:-$HERE/../libbrp_cuda.so}
NVCC=${NVCC:-nvcc}
TMP=$(mktemp -d)
trap 'rm -rf "$TMP"' EXIT
FLAGS="-gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -std=c++17 -Xcompiler -fPIC,-ffp-contract=off"
PIDS=""
for f in api autotune plan fused_kernels fused_fast fused_tc harmonic_fast pass1_warp plain_kernels static_search toplist_filter whiten; do
  $NVCC $FLAGS -c "$HERE/$f.cu" -o "$TMP/$f.o" &
  PIDS="$PIDS $!"
done
g++ -std=c++17 -O2 -fPIC -ffp-contract=off -Wall -Wextra -c "$HERE/host.cpp" -o "$TMP/host.o" &
PIDS="$PIDS $!"
FAIL=0
for p in $PIDS; do wait "$p" || FAIL=1; done
[ "$FAIL" = 0 ] || { echo "build.sh: compilation failed" >&2; exit 1; }
$NVCC -shared -gencode arch=compute_100a,code=sm_100a -o "$OUT.tmp" "$TMP"/*.o
mv "$OUT.tmp" "$OUT"
