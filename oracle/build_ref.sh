#!/usr/bin/env bash
# Test infrastructure only.  Builds the reference's own OpenCL kernels
# (ConvexCell.cl, knearests.cl) as C++ for the host CPU into
# oracle/_ref/libref_kernels.so: the checker for the oracle restatement and
# the timed CPU baseline.  Reads the reference sources where they lie and
# writes nothing but build outputs under oracle/_ref/.
#
# The sources are streamed to g++ with one textual substitution, of
# ConvexCell.cl:45 (`#define make_real4 (real4)`, an OpenCL vector literal that
# is not valid C++), for a call of the shim's constructor function.  No copy
# of the sources is written anywhere.
#
# Usage: build_ref.sh REFERENCE_DIR   (or RPD_REFERENCE_DIR in the environment)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${RPD_REFERENCE_DIR:-}}"
OUT="$HERE/_ref"
if [ -z "$REF" ]; then
  echo "build_ref.sh: no reference directory given (argument or RPD_REFERENCE_DIR); skipping" >&2
  exit 0
fi
if [ ! -f "$REF/ConvexCell.cl" ] || [ ! -f "$REF/knearests.cl" ]; then
  echo "build_ref.sh: reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
# The system g++ (the image also sets $CXX to a toolchain without libgomp).
CXX="${RPD_HOST_CXX:-/usr/bin/g++}"
FLAGS=(-std=c++17 -O2 -fPIC -fopenmp -ffp-contract=off -fno-fast-math -w
       -D__OPENCL_VERSION__=120 -I"$HERE/shim" -I"$REF")

cell() {  # name real vhs grid outdomain [used-cell distance] [hessian components]
  local name=$1 real=$2 vhs=$3 grid=$4 outd=$5 used=${6:-} hc=${7:-}
  local defs=(-DREF_REAL=$real -DVHSAlgo=$vhs -DREF_CELL_ENTRY=ref_cell_$name)
  [ "$real" = double ] && defs+=(-DREF_IS_DOUBLE=1)
  [ "$grid" = 1 ] && defs+=(-DUSE_GRID)
  [ "$outd" = 1 ] && defs+=(-DGRID_OUT_DOMAIN)
  [ -n "$used" ] && defs+=(-DCUSED_CELL -DCUSED_CELL_DIST=$used)
  [ -n "$hc" ] && defs+=(-DCHESSIAN -DHC=$hc)
  { echo '#include "cl_prelude.h"'
    echo '#include "Status.h"'
    echo "namespace ref_cell_ns_$name {"
    echo "#line 1 \"$REF/ConvexCell.cl\""
    sed 's/^#  define make_real4 (real4)$/#  define make_real4 real4_make/' "$REF/ConvexCell.cl"
    echo '#include "ref_cell_adapter.inc"'
    echo '}'
  } | "$CXX" "${FLAGS[@]}" "${defs[@]}" -x c++ -c - -o "$OUT/obj/cell_$name.o"
}
knn() {  # name real
  local name=$1 real=$2
  local defs=(-DREF_REAL=$real -DREF_KNN_ENTRY=ref_knn_$name)
  [ "$real" = double ] && defs+=(-DREF_IS_DOUBLE=1)
  { echo '#include "cl_prelude.h"'
    echo "namespace ref_knn_ns_$name {"
    echo "#line 1 \"$REF/knearests.cl\""
    cat "$REF/knearests.cl"
    echo '#include "ref_knn_adapter.inc"'
    echo '}'
  } | "$CXX" "${FLAGS[@]}" "${defs[@]}" -x c++ -c - -o "$OUT/obj/knn_$name.o"
}

pids=()
for v in 0 1 2; do
  cell f${v}_nogrid float $v 0 0 & pids+=($!)
  cell f${v}_grid float $v 1 0 & pids+=($!)
  cell f${v}_gridout float $v 1 1 & pids+=($!)
done
cell d_nogrid double 2 0 0 & pids+=($!)
cell d_grid double 2 1 0 & pids+=($!)
cell d_gridout double 2 1 1 & pids+=($!)
# used cells (voronoi.cpp:930-939): main passes with distance 0 or 1, and
# the bordering kernel of distances 2 and 3 (no grid)
cell d_grid_used0 double 2 1 0 0 & pids+=($!)
cell d_grid_used1 double 2 1 0 1 & pids+=($!)
cell d_gridout_used1 double 2 1 1 1 & pids+=($!)
cell d_border2 double 2 0 0 2 & pids+=($!)
cell d_border3 double 2 0 0 3 & pids+=($!)
# --hessian (voronoi.cpp:930-936): HC 1 and 4, with and without a grid
for hc in 1 4; do
  cell d_nogrid_h$hc double 2 0 0 "" $hc & pids+=($!)
  cell d_grid_h$hc double 2 1 0 "" $hc & pids+=($!)
  cell d_gridout_h$hc double 2 1 1 "" $hc & pids+=($!)
done
knn f float & pids+=($!)
knn d double & pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
"$CXX" -shared -fopenmp -o "$OUT/libref_kernels.so" "$OUT"/obj/*.o
echo "build_ref.sh: built $OUT/libref_kernels.so"
