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
#
# Build recipe follows the reference's src/CMakeLists.txt:33-36 source list
# with WITH_SIBC, minus mur.c which surface.c:42 #includes.
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
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
  if [ "$mode" = "f64dump" ]; then
    sed -i 's/%16\.8e/%23.16e/g' "$dir/observer.c"
  fi
  local objs=""
  for s in $SRCS; do
    gcc -std=c99 -DNDEBUG -DWITH_SIBC "$@" -I"$REF/uthash" -I"$dir" -c "$dir/$s" -o "$dir/${s%.c}.o"
    objs="$objs $dir/${s%.c}.o"
  done
  gcc "$@" -o "$OUT/$name" $objs -lm
  echo "built $OUT/$name"
}

build_variant vulture_ref_f32          none    -O2
build_variant vulture_oracle_f64       f64     -O2
build_variant vulture_oracle_f64_dump  f64dump -O2
build_variant vulture_ref_f32_omp      none    -O3 -march=x86-64-v3 -fopenmp -DWITH_OPENMP
build_variant vulture_oracle_f64_omp   f64     -O3 -march=x86-64-v3 -fopenmp -DWITH_OPENMP
