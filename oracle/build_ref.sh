#!/usr/bin/env bash
# Build the reference's own CUDA executables for sm_100a, straight from the
# reference sources where they lie (nothing is copied into this repository),
# with the flags of the reference Makefiles (simba/Makefile:8, vfb/Makefile:6)
# except the architecture.  Outputs go to oracle/_ref/ only.
#
#   oracle/_ref/simba_nocache   <- simba/src/nocache.cu + simba/src/instance.cpp
#   oracle/_ref/simba_rtid      <- simba/src/nocache_rtid.cu + simba/src/instance.cpp
#   oracle/_ref/vfb_full_cache  <- vfb/src/full-cache.cu
#
# Usage: oracle/build_ref.sh [path-to-reference]   (default /root/reference)
set -euo pipefail
REF="${1:-/root/reference}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
NVCC="${NVCC:-nvcc}"
ARCH="${CUDA_ARCH:-sm_100a}"
mkdir -p "$OUT"
if [ ! -d "$REF/simba/src" ]; then
  echo "reference sources not found at $REF" >&2
  exit 1
fi
if [ ! -x "$OUT/simba_nocache" ] || [ "$REF/simba/src/nocache.cu" -nt "$OUT/simba_nocache" ]; then
  "$NVCC" -O2 -std=c++20 --extended-lambda -arch="$ARCH" \
    "$REF/simba/src/nocache.cu" "$REF/simba/src/instance.cpp" -o "$OUT/simba_nocache"
fi
if [ ! -x "$OUT/simba_rtid" ] || [ "$REF/simba/src/nocache_rtid.cu" -nt "$OUT/simba_rtid" ]; then
  "$NVCC" -O2 -std=c++20 --extended-lambda -arch="$ARCH" \
    "$REF/simba/src/nocache_rtid.cu" "$REF/simba/src/instance.cpp" -o "$OUT/simba_rtid"
fi
if [ ! -x "$OUT/vfb_full_cache" ] || [ "$REF/vfb/src/full-cache.cu" -nt "$OUT/vfb_full_cache" ]; then
  "$NVCC" -O2 -std=c++20 -I"$REF/vfb/include" -I"$REF/vfb/src" --extended-lambda -arch="$ARCH" \
    "$REF/vfb/src/full-cache.cu" -o "$OUT/vfb_full_cache" 2>&1 | grep -v -i warning || true
fi
ls -la "$OUT"
