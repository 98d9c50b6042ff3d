#!/usr/bin/env bash
# Build the reference's own CUDA executables for sm_100a, straight from the
# reference sources where they lie (nothing is copied into this repository),
# with the flags of the reference Makefiles (simba/Makefile:8, vfb/Makefile:6)
# except the architecture.  Outputs go to oracle/_ref/ only.
#
#   oracle/_ref/simba_nocache      <- simba/src/nocache.cu + simba/src/instance.cpp
#   oracle/_ref/simba_rtid         <- simba/src/nocache_rtid.cu + simba/src/instance.cpp
#   oracle/_ref/vfb_full_cache     <- vfb/src/full-cache.cu
#   oracle/_ref/simba_nocache_u64  <- the same simba sources widened to 64-bit words
#
# The widened build: the reference computes in uint32_t only (samples in
# simba/src/globals.cuh:11-12, the evaluation stack in simba/src/mba.cuh:8,24,
# the instance vectors in simba/src/instance.h:12-13, the JSON reader in
# simba/src/instance.cpp:14-22 and the copy sizes in simba/src/nocache.cu:
# 217,219).  Every `uint32_t` of those five files (and of mba.cuh's unused
# evaluateRPN) becomes `uint64_t` in a scratch copy under $TMPDIR, which is
# compiled and then deleted; nothing else changes (limits, operator order,
# count table, unranking, launch loop).  This is the mechanical widening the
# 64-bit parity fixtures and the 64-bit reference benchmark arm run.
#
# Usage: oracle/build_ref.sh [path-to-reference]
# (or SIMBA_REFERENCE=path); exits 0 without building when neither is given
# and the reference checkout is not at its usual place in the build container.
set -euo pipefail
REF="${1:-${SIMBA_REFERENCE:-/root/reference}}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
NVCC="${NVCC:-nvcc}"
ARCH="${CUDA_ARCH:-sm_100a}"
if [ ! -d "$REF/simba/src" ]; then
  echo "reference sources not found at $REF; reference executables not built" >&2
  exit 0
fi
mkdir -p "$OUT"
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
if [ ! -x "$OUT/simba_nocache_u64" ] || [ "$REF/simba/src/nocache.cu" -nt "$OUT/simba_nocache_u64" ] \
   || [ "$0" -nt "$OUT/simba_nocache_u64" ]; then
  W="$(mktemp -d)"
  trap 'rm -rf "$W"' EXIT
  for f in globals.cuh mba.cuh instance.h instance.cpp nocache.cu; do
    sed 's/\buint32_t\b/uint64_t/g' "$REF/simba/src/$f" > "$W/$f"
  done
  # untouched: the error-check helper and the JSON library
  cp "$REF/simba/src/utils.cuh" "$REF/simba/src/json.hpp" "$W/"
  if grep -q 'uint32_t' "$W/globals.cuh" "$W/mba.cuh" "$W/instance.h" "$W/instance.cpp" "$W/nocache.cu"; then
    echo "widening left a uint32_t behind" >&2
    exit 1
  fi
  "$NVCC" -O2 -std=c++20 --extended-lambda -arch="$ARCH" \
    "$W/nocache.cu" "$W/instance.cpp" -o "$OUT/simba_nocache_u64"
fi
ls -la "$OUT"
