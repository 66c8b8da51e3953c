#!/bin/bash
# TEST INFRASTRUCTURE ONLY.  Builds the reference's own CUDA program for sm_100a
# into oracle/_ref/ (git-ignored; travels to the GPU machine with the tree):
#   oracle/_ref/knnjoin_ref   the reference's knnjoin (src/knnjoin.cu)
#   oracle/_ref/ref_shim.so   the LD_PRELOAD interposer of oracle/ref_shim.c
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or KNN_REFERENCE_ROOT in the
# environment): the root of a checkout of the reference (src/, include/).
#
# The sources are compiled from a temporary copy outside this repository with
# two changes (below): getPoint (include/common8.h:27) is
# declared __host__ __device__ but reads the host global `dim`, which nvcc
# rejects ("identifier dim is undefined in device code"); it is only called
# from host code, so the qualifiers are dropped.  Flags follow the reference's
# Makefile (-w -std=c++11 -O3 -fopenmp -lcublas) with sm_100a for sm_35 and
# the CUDA runtime linked dynamically so that ref_shim.so can interpose.
set -euo pipefail
REF=${1:-${KNN_REFERENCE_ROOT:-}}
if [ -z "$REF" ]; then
  echo "usage: $0 REFERENCE_ROOT (or set KNN_REFERENCE_ROOT)" >&2
  exit 2
fi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
mkdir -p "$OUT"
TMP=$(mktemp -d)
trap 'rm -rf "$TMP"' EXIT
mkdir -p "$TMP/src" "$TMP/include"
cp "$REF/src/knnjoin.cu" "$TMP/src/"
cp "$REF/include/common8.h" "$TMP/include/"
sed -i 's/^inline __host__ __device__ float \* getPoint(/inline float * getPoint(/' \
  "$TMP/include/common8.h"
grep -q '^inline float \* getPoint(' "$TMP/include/common8.h"
# Second change: the context warm-up thread `void *work(void *para)`
# (src/knnjoin.cu:980-982) falls off the end of a non-void function.  g++ 13
# at -O3 emits no return instruction for it, so the thread runs into the next
# function and the process dies with SIGSEGV before printing anything (seen on
# the first run).  It gets the missing `return 0;`.
sed -i '/^void \*work(void \*para){/{n;s/cudaFree(0);/cudaFree(0); return 0;/}' \
  "$TMP/src/knnjoin.cu"
grep -q 'cudaFree(0); return 0;' "$TMP/src/knnjoin.cu"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
CC=/usr/bin/gcc
[ -x "$CC" ] || CC=gcc
"$NVCC" -w -gencode arch=compute_100a,code=sm_100a -std=c++11 -O3 -Xcompiler -fopenmp \
  -I"$TMP/include" "$TMP/src/knnjoin.cu" -o "$OUT/knnjoin_ref" -lcublas -lgomp -cudart shared
"$CC" -O2 -fPIC -shared -o "$OUT/ref_shim.so" "$HERE/ref_shim.c" -ldl
echo "$OUT/knnjoin_ref"
