#!/bin/sh
# Compiles the reference's own sources, unchanged, from where they lie under
# the reference tree (strict IEEE flags, as for the parity oracle):
#   oracle/_ref/libref.so      the formula files, camera, projection, RNG and
#                              algebra with oracle/ref_harness.cpp
#   oracle/_ref/librefpipe.so  every formula of formula/definition/ and the
#                              path's src/ files (parameters, objects tree,
#                              sequences, Compute, CalculateDistance, the
#                              render worker and its shaders, cImage) with
#                              oracle/ref_pipeline.cpp, against the Qt
#                              stand-ins of oracle/ref_shim/
# Needs the reference tree; the product never uses the results.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
MB=${MB:-/root/reference/mandelbulber2}
OUT="$HERE/_ref"
if [ ! -d "$MB/src" ]; then
  echo "reference tree not found at $MB; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
CXX=${CXX:-g++}
JOBS=${JOBS:-$(nproc 2>/dev/null || echo 4)}
FLAGS="-std=c++17 -O2 -fno-fast-math -ffp-contract=off -fPIC -w -I$MB -I$MB/src -I$MB/formula/definition -I$HERE/ref_shim"
SRCS="$MB/formula/definition/fractal_mandelbulb.cpp $MB/formula/definition/fractal_mandelbox.cpp \
$MB/formula/definition/fractal_menger_sponge.cpp $MB/formula/definition/fractal_mandelbulb_power2.cpp \
$MB/formula/definition/fractal_hypercomplex.cpp $MB/formula/definition/fractal_kaleidoscopic_ifs.cpp $MB/formula/definition/fractal_xenodreambuie.cpp \
$MB/src/camera_target.cpp $MB/src/projection_3d.cpp \
$MB/src/common_math.cpp $MB/src/algebra.cpp $HERE/ref_harness.cpp"
if [ ! -f "$OUT/libref.so" ] || [ -n "$(find $HERE/ref_harness.cpp $HERE/ref_shim -newer "$OUT/libref.so" 2>/dev/null)" ]; then
  $CXX $FLAGS -shared -o "$OUT/libref.so" $SRCS
  echo "built $OUT/libref.so"
fi

# the pipeline library: one object per source, compiled in parallel
PIPE_SRC="compute_fractal calculate_distance parameters one_parameter multi_val initparameters fractal \
fractparams hybrid_fractal_sequences objects_tree primitives primitive fractal_container fractal_coloring \
orbit_trap_shape common_math algebra camera_target projection_3d light lights statistics histogram material \
rendering_configuration perlin_noise_octaves displacement_map texture_mapping color_gradient stereo \
shader_perlin_noise_for_shaders render_worker cimage scheduler hsv2rgb"
LIST="$OUT/obj/sources.txt"
: > "$LIST"
for f in $PIPE_SRC; do echo "$MB/src/$f.cpp" >> "$LIST"; done
for f in $MB/src/shader_*.cpp $MB/formula/definition/*.cpp; do
  case "$f" in *shader_perlin_noise_for_shaders.cpp) ;; *) echo "$f" >> "$LIST" ;; esac
done
NEWEST=$(ls -t $HERE/ref_shim/qshim_core.h $HERE/ref_pipeline.cpp $HERE/ref_pipeline_stubs.cpp | head -1)
sort -u "$LIST" | while read -r src; do
  obj="$OUT/obj/$(echo "$src" | sed "s|^$MB/||; s|/|_|g; s|\.cpp$|.o|")"
  if [ ! -f "$obj" ] || [ "$src" -nt "$obj" ] || [ "$HERE/ref_shim/qshim_core.h" -nt "$obj" ]; then
    echo "$src $obj"
  fi
done | xargs -r -P "$JOBS" -n 2 sh -c "$CXX $FLAGS -c \"\$0\" -o \"\$1\""
$CXX $FLAGS -c "$HERE/ref_pipeline.cpp" -o "$OUT/obj/_ref_pipeline.o"
$CXX $FLAGS -c "$HERE/ref_pipeline_stubs.cpp" -o "$OUT/obj/_ref_pipeline_stubs.o"
$CXX -shared -o "$OUT/librefpipe.so" "$OUT"/obj/*.o
echo "built $OUT/librefpipe.so"
