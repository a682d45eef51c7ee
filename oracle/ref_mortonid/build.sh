#!/bin/bash
# Compiles the reference's own Morton-id code (src/mortonid.cpp,
# include/mortonid.{hpp,txx}) from the read-only reference tree into
# oracle/_ref/libmortonid_ref.so.  Only the golden-vector script uses it.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${PVFMM_REFERENCE:-/root/reference}"
OUT="$HERE/../_ref"
if [ ! -d "$REF/src" ] || [ ! -d "$REF/include" ]; then
  echo "reference sources not found at $REF: checker not built"
  exit 0
fi
mkdir -p "$OUT"
g++ -O2 -std=c++17 -shared -fPIC -I "$HERE/shim" -I "$REF/include" \
    "$REF/src/mortonid.cpp" "$HERE/mortonid_wrap.cpp" -o "$OUT/libmortonid_ref.so"
