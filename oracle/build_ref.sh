#!/bin/sh
# Builds the parts of the reference that compile from their own sources
# without Eigen (only core/math/legendre.h) into oracle/_ref/.  Needs the
# reference tree at $MRTRIX_REF (default /root/reference); skipped without it.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${MRTRIX_REF:-/root/reference}
if [ ! -f "$REF/core/math/legendre.h" ]; then
  echo "reference tree not found at $REF; oracle/_ref not built" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++11 -fPIC -shared -I "$HERE/ref_stub" -I "$REF/core" \
    "$HERE/ref_legendre_shim.cpp" -o "$HERE/_ref/libref_legendre.so"
echo "built $HERE/_ref/libref_legendre.so"
