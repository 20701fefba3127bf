#!/bin/sh
# Builds libbrp_cuda.so in this directory's parent (the package root) for sm_100a.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=${1:-$HERE/../libbrp_cuda.so}
NVCC=${NVCC:-nvcc}
TMP=$(mktemp -d)
trap 'rm -rf "$TMP"' EXIT
FLAGS="-gencode arch=compute_100a,code=sm_100a -lineinfo -O3 -std=c++17 -Xcompiler -fPIC,-ffp-contract=off"
for f in api plan fused_kernels plain_kernels; do
  $NVCC $FLAGS -c "$HERE/$f.cu" -o "$TMP/$f.o" &
done
g++ -std=c++17 -O2 -fPIC -ffp-contract=off -Wall -Wextra -c "$HERE/host.cpp" -o "$TMP/host.o" &
wait
$NVCC -shared -gencode arch=compute_100a,code=sm_100a -o "$OUT" "$TMP"/*.o
