#!/usr/bin/env bash
# Builds the reference's own code, straight from its source tree, into
# oracle/_ref/libmr_ref.so for the parity tests (test infrastructure only).
# The three baseline-reorderer headers the reference includes are replaced by
# the stand-ins in oracle/ref_stubs/ (their libraries need boost, libnuma and
# a network fetch). Nothing is copied out of the reference tree.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
# the reference checkout sits beside this repository unless MR_REFERENCE_DIR names it
REF=${MR_REFERENCE_DIR:-$(dirname "$(dirname "$HERE")")/reference}
OUT="$HERE/_ref"
if [ ! -f "$REF/src/class.cu" ]; then
  echo "build_ref: reference sources not found at $REF; nothing built"
  exit 0
fi
mkdir -p "$OUT"
if [ "$OUT/libmr_ref.so" -nt "$HERE/ref_shim.cu" ] && [ "$OUT/libmr_ref.so" -nt "$REF/src/class.cu" ]; then
  echo "build_ref: up to date"
  exit 0
fi
nvcc -std=c++17 -O2 --extended-lambda -w -Xcompiler -fPIC,-fopenmp -shared \
  -gencode arch=compute_100a,code=sm_100a -lineinfo \
  -I"$HERE/ref_stubs" -I"$REF/include" -DREF_CLASS_CU="\"$REF/src/class.cu\"" \
  "$HERE/ref_shim.cu" "$HERE/ref_stubs/stubs.cpp" -o "$OUT/libmr_ref.so.tmp" \
  -lcusparse -lcublas -lgomp
mv "$OUT/libmr_ref.so.tmp" "$OUT/libmr_ref.so"
echo "build_ref: built $OUT/libmr_ref.so"
