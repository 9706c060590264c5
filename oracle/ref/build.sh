#!/bin/bash
# Compiles the reference's own CUDA libraries (lib/**/*.cu, from the sources where they lie under
# the reference tree, never copied) plus oracle/ref/ref_driver.cu into oracle/_ref/libref.so.
# TEST INFRASTRUCTURE ONLY: used to check parity with, and to time, the reference build.
set -euo pipefail
REF=${REFERENCE_ROOT:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/../_ref
[ -d "$REF/lib" ] || { echo "reference tree not found at $REF"; exit 0; }
mkdir -p "$OUT/obj"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
INC="-I$REF/lib/force_model/include -I$REF/lib/common/gpu_utils/include -I$REF/lib/common/gpu_constants \
-I$REF/lib/common/types -I$REF/lib/gpu_startup/include -I$REF/lib/gpu_integrator/include \
-I$REF/lib/gpu_propagator/include -I$REF/lib/closest_approach/include"
FLAGS="-std=c++20 -O3 -rdc=true --expt-relaxed-constexpr -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -w"
SRCS=$(cd "$REF" && find lib/force_model lib/gpu_startup lib/gpu_integrator lib/gpu_propagator lib/closest_approach -name '*.cu' | sort)
OBJS=""
for s in $SRCS; do
  o="$OUT/obj/$(echo "$s" | tr '/' '_' | sed 's/\.cu$/.o/')"
  if [ ! -f "$o" ] || [ "$REF/$s" -nt "$o" ]; then
    $NVCC $FLAGS $INC -c "$REF/$s" -o "$o" &
  fi
  OBJS="$OBJS $o"
done
wait
$NVCC $FLAGS $INC -c "$HERE/ref_driver.cu" -o "$OUT/obj/ref_driver.o"
$NVCC -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fPIC -o "$OUT/libref.so" $OBJS "$OUT/obj/ref_driver.o" -lcublas -lcudart
echo "built $OUT/libref.so"
