#!/usr/bin/env bash
# Builds oracle/_ref/libref.so: the reference's own kernels and host routines,
# compiled unchanged from the reference tree through oracle/ref_shim, plus
# oracle/ref_driver.cpp (the dispatch order of Compute.cpp).  Nothing is copied
# out of the reference; outputs go only to oracle/_ref/ (git-ignored).
# Usage: oracle/ref_build.sh [reference root, default /root/reference]
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${SPH_REFERENCE_ROOT:-/root/reference}}/SPH"
SH="$REF/Shaders"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
if [ ! -d "$SH" ]; then echo "reference sources not found under $REF" >&2; exit 2; fi
mkdir -p "$OBJ"
CXX="${SPH_HOST_CXX:-g++}"
COMMON=(-O3 -fPIC -fopenmp -ffp-contract=off -fno-fast-math -std=c++17 -w)
MSL=(-x c++ -fsingle-precision-constant -Wno-attributes -I "$HERE/ref_shim" -I "$SH")
objs=()
for f in sort density accelerations step gravity/gravity gravity/poles/P2M gravity/poles/M2M \
         gravity/poles/M2L gravity/poles/L2L gravity/poles/L2P gravity/poles/derivatives \
         gravity/poles/accept gravity/poles/helpers render; do
  o="$OBJ/$(echo "$f" | tr '/' '_').o"
  "$CXX" "${COMMON[@]}" "${MSL[@]}" -c "$SH/$f.metal" -o "$o"
  objs+=("$o")
done
"$CXX" "${COMMON[@]}" -I "$HERE/ref_shim" -I "$REF" -c "$REF/octree/octree.cpp" -o "$OBJ/octree.o"
"$CXX" "${COMMON[@]}" -I "$HERE/ref_shim" -I "$REF/Buffers" -I "$REF" -c "$REF/ANEOS/ANEOS.cpp" -o "$OBJ/ANEOS.o"
"$CXX" "${COMMON[@]}" -fsingle-precision-constant -Wno-attributes -I "$HERE" -I "$HERE/ref_shim" \
  -I "$SH/gravity/poles" -c "$HERE/ref_driver.cpp" -o "$OBJ/ref_driver.o"
"$CXX" -shared -fopenmp -o "$OUT/libref.so" "${objs[@]}" "$OBJ/octree.o" "$OBJ/ANEOS.o" "$OBJ/ref_driver.o"
echo "built $OUT/libref.so"
