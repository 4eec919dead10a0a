#!/bin/bash
# Builds oracle/_ref/libref.so: the reference's host operator surface
# (oapUtils, oapMath, oapMatrix, oapMatrixCpu compiled from the reference
# sources where they lie, unchanged) plus ref_driver.cpp's C entry points.
# Test infrastructure only; outputs go to oracle/_ref/ (git-ignored).
set -euo pipefail
# The oap checkout: $OAP_REFERENCE, else the first argument, else the
# location this build's container mounts it at.  Without a checkout there is
# nothing to build (the GPU box uses the prebuilt library).
REF=${OAP_REFERENCE:-${1:-/root/reference}}
if [ ! -d "$REF/oapMatrixCpu" ]; then
  echo "no oap checkout at $REF; oracle/_ref not built"
  exit 0
fi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/../_ref"
OBJ="$OUT/obj"
mkdir -p "$OBJ"
INC="-I$REF/oapUtils -I$REF/oapMath -I$REF/oapMatrix -I$REF/oapMatrixCpu -I$REF/oapMatrixCuda -I$REF/oapCuda -I$REF/ArnoldiPackage"
FLAGS="-std=c++11 -O2 -fPIC -DOAP_CONFIG_NI_EF -DOAP_PATH=\"$REF\" -DTMP_PATH=\"/tmp/Oap\""
objs=()
for dir in oapUtils oapMath oapMatrix oapMatrixCpu; do
  for src in "$REF/$dir"/*.cpp; do
    o="$OBJ/${dir}_$(basename "$src" .cpp).o"
    if [ ! -f "$o" ] || [ "$src" -nt "$o" ] || [ "$0" -nt "$o" ]; then
      g++ $FLAGS $INC -w -c "$src" -o "$o"
    fi
    objs+=("$o")
  done
done
g++ $FLAGS $INC -c "$HERE/ref_driver.cpp" -o "$OBJ/ref_driver.o"
g++ -shared -o "$OUT/libref.so" "$OBJ/ref_driver.o" "${objs[@]}" -lpthread
echo "built $OUT/libref.so"
