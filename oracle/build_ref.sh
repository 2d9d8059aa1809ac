#!/bin/sh
# Compiles the reference's own sources for the hot path's formulas, camera
# and RNG (unchanged, from where they lie under the reference tree) together
# with oracle/ref_harness.cpp into oracle/_ref/libref.so.  Strict IEEE flags,
# as for the parity oracle.  Needs the reference tree; the product never
# uses the result.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
MB=${MB:-/root/reference/mandelbulber2}
OUT="$HERE/_ref"
if [ ! -d "$MB/src" ]; then
  echo "reference tree not found at $MB; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$OUT"
CXX=${CXX:-g++}
FLAGS="-std=c++17 -O2 -fno-fast-math -ffp-contract=off -fPIC -I$MB -I$MB/src -I$MB/formula/definition -I$HERE/ref_shim"
SRCS="$MB/formula/definition/fractal_mandelbulb.cpp $MB/formula/definition/fractal_mandelbox.cpp \
$MB/formula/definition/fractal_menger_sponge.cpp $MB/formula/definition/fractal_mandelbulb_power2.cpp \
$MB/formula/definition/fractal_hypercomplex.cpp $MB/formula/definition/fractal_kaleidoscopic_ifs.cpp $MB/formula/definition/fractal_xenodreambuie.cpp \
$MB/src/camera_target.cpp $MB/src/projection_3d.cpp \
$MB/src/common_math.cpp $MB/src/algebra.cpp $HERE/ref_harness.cpp"
$CXX $FLAGS -shared -o "$OUT/libref.so" $SRCS
echo "built $OUT/libref.so"
