#!/usr/bin/env bash
# Builds the reference's own time-step code (LBM-C solver.cu, collision.cu,
# boundary_conditions/**, macros.cu, data_types.cuh) as host C++ shared
# objects for the oracle.  TEST INFRASTRUCTURE ONLY.
#
#   oracle/_ref/libref_d2q9_asis.so     D2Q9, reference as is
#   oracle/_ref/libref_d2q9_patched.so  D2Q9, Smagorinsky q_bar zero-initialised
#   oracle/_ref/libref_d3q15_asis.so    D3Q15, reference as is
#   oracle/_ref/libref_reader_{d2q9,d3q15}.so  the input-file reader
#       (infile_reader.cu) for each lattice, unpatched
#   oracle/_ref/libref_d3q15_patched.so D3Q15 with the documented fixes:
#       macros.cu:97-115  M_inv integer divisions -> floating point
#       collision.cu:492-496  (-7/3) -> (-7.0/3.0)
#       collision.cu:447  q_bar zero-initialised
#       d3q15_zh_defs.cu:87-91  zh_pressure_Z uses u[2] (the z velocity)
#
# The lattice is chosen at compile time in the reference (macros.cu:11-12),
# so the D2Q9 builds and the patched builds compile a temporary edited copy
# of the needed files from oracle/_ref/gen/, which is deleted after the
# build; only the .so files stay.  Nothing is copied into the repository.
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT
#    or: LBMC_REFERENCE_ROOT=... oracle/build_ref.sh
# REFERENCE_ROOT is the directory that holds the reference's LBM-C/ folder.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT_ARG="${1:-${LBMC_REFERENCE_ROOT:-}}"
if [ -z "$ROOT_ARG" ]; then
  echo "build_ref: give the reference root as an argument or in LBMC_REFERENCE_ROOT" >&2
  exit 2
fi
REF="$ROOT_ARG/LBM-C"
OUT="$HERE/_ref"
if [ ! -f "$REF/solver.cu" ]; then
  echo "build_ref: reference sources not found at $REF" >&2
  exit 2
fi
mkdir -p "$OUT"
CXX="${ORACLE_CXX:-/usr/bin/g++}"
FLAGS="-O2 -fopenmp -fPIC -shared -fpermissive -w -ffp-contract=off -fno-fast-math"

build_variant() {
  local lat="$1" variant="$2"
  local gen="$OUT/gen/${lat}_${variant}"
  rm -rf "$gen"
  mkdir -p "$gen/boundary_conditions/d2q9" "$gen/boundary_conditions/d3q15"
  for f in macros.cu data_types.cuh solver.cu solver.cuh collision.cu collision.cuh infile_reader.cu; do
    cp "$REF/$f" "$gen/$f"
  done
  for f in macro_bc.cu macro_bc.cuh micro_bc.cuh \
           d2q9/d2q9_sf_defs.cu d2q9/d2q9_sf_defs.cuh d2q9/d2q9_zh_defs.cu d2q9/d2q9_zh_defs.cuh \
           d3q15/d3q15_sf_defs.cu d3q15/d3q15_sf_defs.cuh d3q15/d3q15_zh_defs.cu d3q15/d3q15_zh_defs.cuh; do
    cp "$REF/boundary_conditions/$f" "$gen/boundary_conditions/$f"
  done
  chmod -R u+w "$gen"
  if [ "$lat" = "d2q9" ]; then
    sed -i 's/^#define D3Q15/#define D2Q9/' "$gen/macros.cu"
  fi
  if [ "$variant" = "patched" ]; then
    # D3Q15 M_inv literals: integer division -> floating point division.
    sed -i '/define LOAD_M_INV/,/memcpy(m_inv_tmp/ s#\([0-9][0-9]*\)/\([0-9][0-9]*\)#\1.0/\2.0#g' "$gen/macros.cu"
    sed -i 's#(-7/3)#(-7.0/3.0)#g' "$gen/collision.cu"
    sed -i 's#double q_bar\[DIM\]\[DIM\];#double q_bar[DIM][DIM] = {};#' "$gen/collision.cu"
    # zh_pressure_Z: the unknowns use the z velocity.
    sed -i '86,92 s#current_node->u\[0\]#current_node->u[2]#g' "$gen/boundary_conditions/d3q15/d3q15_zh_defs.cu"
  fi
  $CXX $FLAGS -I "$gen" -I "$HERE/shim_include" "$HERE/ref_shim.cpp" \
      -o "$OUT/libref_${lat}_${variant}.so"
  if [ "$variant" = "asis" ]; then
    # The input-file reader (infile_reader.cu), unpatched.
    $CXX $FLAGS -I "$gen" -I "$HERE/shim_include" "$HERE/ref_reader_shim.cpp" \
        -o "$OUT/libref_reader_${lat}.so"
    echo "built $OUT/libref_reader_${lat}.so"
  fi
  rm -rf "$gen"
  echo "built $OUT/libref_${lat}_${variant}.so"
}

for lat in d2q9 d3q15; do
  for variant in asis patched; do
    build_variant "$lat" "$variant"
  done
done
rmdir "$OUT/gen" 2>/dev/null || true
