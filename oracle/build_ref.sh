#!/bin/sh
# Compile the reference's own ring-table, Legendre, spin-weighted Wigner-d and pixel-coordinate
# kernels (ring_tables_healpix.cu, legendre.cu, wigner_d_ms.cu, coords_ring.cu, nested_gpu.cu,
# nested_pix2ang.cu) as host C++ straight from the reference tree, into oracle/_ref/libhbref.so.
# Test infrastructure only; nothing is copied out of the reference tree.
set -e
REF=${1:-${HB_REFERENCE_DIR:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -f "$REF/ring_tables_healpix.cu" ]; then
  echo "reference tree not found at $REF; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$OUT"
CXX=${CXX:-g++}
for f in ring_tables_healpix legendre wigner_d_ms coords_ring nested_gpu nested_pix2ang; do
  $CXX -O2 -fPIC -std=c++17 -include "$HERE/ref_prelude.h" -x c++ -c "$REF/$f.cu" -o "$OUT/$f.o"
done
$CXX -O2 -fPIC -std=c++17 -I"$HERE" -c "$HERE/ref_launch.cpp" -o "$OUT/ref_launch.o"
$CXX -shared -o "$OUT/libhbref.so" "$OUT/ring_tables_healpix.o" "$OUT/legendre.o" "$OUT/wigner_d_ms.o" "$OUT/coords_ring.o" "$OUT/nested_gpu.o" \
  "$OUT/nested_pix2ang.o" "$OUT/ref_launch.o"
rm -f "$OUT"/*.o
echo "built $OUT/libhbref.so"
