#!/bin/sh
# ORACLE TEST INFRASTRUCTURE: compiles the reference's own shader sources
# (read from the reference checkout: $DSPBR_REFERENCE, else the directory
# "reference" beside this repository) as C++ into
# oracle/_ref/ (git-ignored).  FP32 and FP64 variants.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ORACLE=$(dirname "$HERE")
REF=${DSPBR_REFERENCE:-$(dirname "$ORACLE")/../reference}
OUT="$ORACLE/_ref"
CXX=${CXX:-g++}
if [ ! -f "$REF/packages/lib/shader/renderer.frag" ]; then
  echo "build_ref: reference shaders not found under $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
for v in f32 f64; do
  if [ "$v" = f64 ]; then FLAG=--fp64; REAL=double; else FLAG=; REAL=float; fi
  python3 "$HERE/glsl2cpp.py" --ref "$REF" --chunks "$HERE/chunks" --out "$OUT/glsl_ref_$v.inc" $FLAG
  python3 "$HERE/glsl2cpp.py" --ref "$REF" --chunks "$HERE/chunks" --out "$OUT/glsl_post_$v.inc" --post $FLAG
  $CXX -std=c++20 -O3 -march=native -ffp-contract=off -fPIC -shared -w \
    -I"$HERE" -I"$OUT" -DGLSL_REAL=$REAL -DREF_PREFIX=ref_${v}_ "-DREF_SOURCE=\"glsl_ref_$v.inc\"" \
    "-DREF_POST_SOURCE=\"glsl_post_$v.inc\"" \
    "$HERE/ref_harness.cpp" -o "$OUT/libglslref_$v.so" -lpthread
done
echo "build_ref: built $OUT/libglslref_f32.so $OUT/libglslref_f64.so"
