#!/usr/bin/env bash
# Build the reference solver (Vulture 0.7.1, C99) from its own sources as the
# oracle's strengthener.  This is test infrastructure: only tests/, the smoke
# check and the CPU-baseline leg of bench.py execute the binaries it makes.
#
# The sources are read where they lie: $VULTURE_REF, by default a checkout
# named `reference` beside this repository.  The
# FP64 variants need three edits to the reference, so those are built from a
# patched copy in a temporary directory outside the repository; nothing from
# the reference is ever written into the repository.  Outputs go to
# oracle/_ref/ only (git-ignored; travels to the GPU host with the tree).
#
# Variants:
#   vulture_ref_f32        as shipped (typedef float real), gcc -O2 -std=c99,
#                          reproduces the reference's golden .asc files.
#   vulture_ref_f32_omp    as shipped, -O3 -fopenmp: the timed CPU baseline.
#   vulture_oracle_f64     real=double, sscanf %e->%le for PML/SIBC cards
#                          (boundary.c:173,184), fdtd_types.h:36-38 DBL_*.
#   vulture_oracle_f64_dump  as above, observer text printed with 17
#                          significant digits (observer.c:791-793,965-983)
#                          so FP64 parity can be checked at 1e-12.
#   vulture_oracle_f64_omp FP64 with OpenMP, for the FP64 CPU baseline.
#   vulture_ref_gpu        as vulture_oracle_f64_dump, but its propagate()
#                          (simulation.c:136-231) is the GPU replacement of
#                          oracle/propagate_gpu/propagate_gpu.c, linked against
#                          vulture_b200/lib/libvulture_b200.so (built first);
#                          getters of the modules' private state are appended
#                          to copies of pml.c, mur.c, source.c and observer.c.
#   vulture_ref_oracle_shim the same replacement on the CPU oracle instead
#                          of the GPU (oracle/propagate_gpu/vgpu_on_oracle.c):
#                          checks the replacement's state mapping with no GPU.
#
# Build recipe follows the reference's src/CMakeLists.txt:33-36 source list
# with WITH_SIBC, minus mur.c which surface.c:42 #includes.
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ONLY="${1:-}"   # build only this variant (default: all)
REF="${VULTURE_REF:-$HERE/../../reference}"
OUT="$HERE/_ref"
mkdir -p "$OUT"

if [ ! -d "$REF/src" ]; then
  echo "reference sources not found at $REF/src" >&2
  exit 1
fi

SRCS="fdtd_types.c physical.c message.c alloc_array.c simulation.c bounding_box.c
      mesh.c grid.c pml.c gnuplot.c gmsh.c timer.c memory.c medium.c block.c
      boundary.c surface.c waveform.c source.c planewave.c observer.c util.c
      debye.c wire.c line.c sibc.c filter.c vulture.c"

TMP="$(mktemp -d /tmp/vulture_oracle.XXXXXX)"
trap 'rm -rf "$TMP"' EXIT

# $1 name, $2 patch mode (none|f64|f64dump), $3.. extra flags
build_variant() {
  local name="$1" mode="$2"; shift 2
  if [ -n "$ONLY" ] && [ "$ONLY" != "$name" ]; then return 0; fi
  local dir="$TMP/$name"
  mkdir -p "$dir"
  cp "$REF"/src/*.c "$REF"/src/*.h "$dir"/
  if [ "$mode" != "none" ]; then
    sed -i 's/^typedef float real;/typedef double real;/;
            s/#define REAL_MAX     FLT_MAX/#define REAL_MAX     DBL_MAX/;
            s/#define REAL_EPSILON FLT_EPSILON/#define REAL_EPSILON DBL_EPSILON/' "$dir/fdtd_types.h"
    grep -q '^typedef double real;' "$dir/fdtd_types.h"
    sed -i '173s/%e %e %e/%le %le %le/; 184s/%e %e %e %e %e %e %e %e/%le %le %le %le %le %le %le %le/' "$dir/boundary.c"
    grep -q '%le %le %le %le %le %le %le %le' "$dir/boundary.c"
  fi
  if [ "$mode" = "f64dump" ] || [ "$mode" = "gpu" ] || [ "$mode" = "shim_on_oracle" ]; then
    sed -i 's/%16\.8e/%23.16e/g' "$dir/observer.c"
  fi
  local extra="" libs=""
  if [ "$mode" = "gpu" ] || [ "$mode" = "shim_on_oracle" ]; then
    sed -i 's/^void propagate( void )$/void propagateCpu( void )/' "$dir/simulation.c"
    grep -q '^void propagateCpu( void )$' "$dir/simulation.c"
    for m in pml mur source observer; do
      cat "$HERE/propagate_gpu/state_$m.inc.c" >> "$dir/$m.c"
    done
    gcc -std=c99 -DNDEBUG -DWITH_SIBC "$@" -I"$REF/uthash" -I"$dir" -I"$HERE/../include" \
        -c "$HERE/propagate_gpu/propagate_gpu.c" -o "$dir/propagate_gpu.o"
    extra="$dir/propagate_gpu.o"
    if [ "$mode" = "gpu" ]; then
      libs="-L$HERE/../vulture_b200/lib -lvulture_b200 -Wl,-rpath,\$ORIGIN/../../vulture_b200/lib"
    else
      gcc -std=gnu11 -O2 -ffp-contract=off -I"$HERE/../include" -c "$HERE/propagate_gpu/vgpu_on_oracle.c" \
          -o "$dir/vgpu_on_oracle.o"
      gcc -std=gnu11 -O2 -ffp-contract=off -I"$HERE/../include" -DVCPU_REAL=double -DVCPU_PREFIX=vcpu64_ \
          -c "$HERE/vcpu.c" -o "$dir/vcpu64.o"
      extra="$extra $dir/vgpu_on_oracle.o $dir/vcpu64.o"
    fi
  fi
  local objs=""
  for s in $SRCS; do
    gcc -std=c99 -DNDEBUG -DWITH_SIBC "$@" -I"$REF/uthash" -I"$dir" -c "$dir/$s" -o "$dir/${s%.c}.o"
    objs="$objs $dir/${s%.c}.o"
  done
  gcc "$@" -o "$OUT/$name" $objs $extra -lm $libs
  echo "built $OUT/$name"
}

build_variant vulture_ref_f32          none    -O2
build_variant vulture_oracle_f64       f64     -O2
build_variant vulture_oracle_f64_dump  f64dump -O2
build_variant vulture_ref_f32_omp      none    -O3 -march=x86-64-v3 -fopenmp -DWITH_OPENMP
build_variant vulture_oracle_f64_omp   f64     -O3 -march=x86-64-v3 -fopenmp -DWITH_OPENMP
build_variant vulture_ref_oracle_shim shim_on_oracle -O2
if [ -f "$HERE/../vulture_b200/lib/libvulture_b200.so" ]; then
  build_variant vulture_ref_gpu        gpu     -O2
fi
