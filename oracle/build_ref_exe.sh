#!/bin/sh
# Build the reference solver as an executable, twice, from its own sources
# compiled where they lie (read-only) with its Makefile flags (Makefile:19),
# plus the GSL / LAPACK stand-ins of oracle/shims:
#   oracle/_ref/field_solver      the reference as shipped (main.C's driver
#                                 over the reference's own solve());
#   oracle/_ref/field_solver_gpu  the same driver with
#                                 flow-solver_b200/shim/solve_gpu.C in place
#                                 of solve.C, and grid_io.C's
#                                 write_surface_cp and Compute_Body_Forces
#                                 made weak so that
#                                 the shim's definitions link (the integration
#                                 a maintainer makes, without editing a
#                                 reference file), linked to libflowgpu.so;
#   oracle/_ref/field_solver_stages  the reference's own solve() with
#                                 build_matrix, build_interior_residuals,
#                                 build_boundary_residuals and linear_solve
#                                 from flow-solver_b200/shim/stages_gpu.C
#                                 (the reference's made weak), linked to
#                                 libflowgpu.so.
# Test infrastructure: tests/test_gpu_dropin_exe.py runs both on one case and
# compares their output files.  Needs flow-solver_b200/lib/libflowgpu.so.
# Usage: sh oracle/build_ref_exe.sh reference_dir   (or FLOW_REFERENCE_DIR=... sh oracle/build_ref_exe.sh)
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-$FLOW_REFERENCE_DIR}
if [ -z "$REF" ]; then
  echo "build_ref_exe.sh: give the reference directory as the argument or in FLOW_REFERENCE_DIR" >&2
  exit 1
fi
OUT="$HERE/_ref"
OBJ="$OUT/exe_obj"
HOST="$HERE/../flow-solver_b200/csrc/host"
LIBDIR="$HERE/../flow-solver_b200/lib"
if [ ! -f "$REF/solve.C" ]; then
  echo "build_ref_exe.sh: reference sources not found at $REF" >&2
  exit 1
fi
if [ ! -f "$LIBDIR/libflowgpu.so" ]; then
  echo "build_ref_exe.sh: build libflowgpu.so first" >&2
  exit 1
fi
mkdir -p "$OBJ"
CFLAGS="-Wno-deprecated -Wall -ansi -pedantic -O3"
INC="-I$REF/include -I$HERE/shims -I$HOST"
for f in "$REF"/*.C; do
  b=$(basename "$f" .C)
  g++ -x c++ $CFLAGS $INC -w -c "$f" -o "$OBJ/$b.o"
done
gcc -O2 -I"$HOST" -c "$HOST/quadrature.c" -o "$OBJ/quadrature.o"
gcc -O2 -I"$HOST" -c "$HOST/svd.c" -o "$OBJ/svd.o"
gcc -O2 -I"$HERE/shims" -I"$HOST" -c "$HERE/shims/gsl_shim.c" -o "$OBJ/gsl_shim.o"
gcc -O2 -I"$HOST" -c "$HERE/shims/lapack_shim.c" -o "$OBJ/lapack_shim.o"
SHIMS="$OBJ/quadrature.o $OBJ/svd.o $OBJ/gsl_shim.o $OBJ/lapack_shim.o"
REFOBJ=""
for f in "$REF"/*.C; do
  b=$(basename "$f" .C)
  [ "$b" = solve ] && continue
  [ "$b" = grid_io ] && continue
  REFOBJ="$REFOBJ $OBJ/$b.o"
done
g++ -o "$OUT/field_solver" $REFOBJ "$OBJ/solve.o" "$OBJ/grid_io.o" $SHIMS -lm
# the two grid_io.C functions the shim replaces, weak in a copy of grid_io.o
WEAK=""
for fn in write_surface_cp Compute_Body_Forces; do
  sym=$(nm "$OBJ/grid_io.o" | awk -v f="$fn" '$2 == "T" && $3 ~ ("^_Z[0-9]+" f "P") {print $3}')
  [ -n "$sym" ] || { echo "build_ref_exe.sh: $fn not found in grid_io.o" >&2; exit 1; }
  WEAK="$WEAK --weaken-symbol=$sym"
done
objcopy $WEAK "$OBJ/grid_io.o" "$OBJ/grid_io_weak.o"
g++ -x c++ $CFLAGS -Wno-long-long $INC -I"$HERE/../include" -c \
    "$HERE/../flow-solver_b200/shim/solve_gpu.C" -o "$OBJ/solve_gpu.o"
g++ -o "$OUT/field_solver_gpu" $REFOBJ "$OBJ/solve_gpu.o" "$OBJ/grid_io_weak.o" $SHIMS \
    -L"$LIBDIR" -lflowgpu -Wl,-rpath,'$ORIGIN/../../flow-solver_b200/lib' -lm
# the reference's own solve() over the stage shim: build_matrix,
# build_interior_residuals, build_boundary_residuals and linear_solve made
# weak in copies of their objects, the shim's definitions linked instead
weaken() {  # object, functions...
  obj=$1; shift
  flags=""
  for fn in "$@"; do
    sym=$(nm "$OBJ/$obj.o" | awk -v f="$fn" '$2 == "T" && $3 ~ ("^_Z[0-9]+" f "P") {print $3}')
    [ -n "$sym" ] || { echo "build_ref_exe.sh: $fn not found in $obj.o" >&2; exit 1; }
    flags="$flags --weaken-symbol=$sym"
  done
  objcopy $flags "$OBJ/$obj.o" "$OBJ/${obj}_weak.o"
}
weaken init_memory build_matrix
weaken residual build_interior_residuals build_boundary_residuals
weaken linear_algebra linear_solve
STAGEOBJ=""
for f in "$REF"/*.C; do
  b=$(basename "$f" .C)
  case "$b" in
    init_memory|residual|linear_algebra) STAGEOBJ="$STAGEOBJ $OBJ/${b}_weak.o" ;;
    *) STAGEOBJ="$STAGEOBJ $OBJ/$b.o" ;;
  esac
done
g++ -x c++ $CFLAGS -Wno-long-long $INC -I"$HERE/../include" -c \
    "$HERE/../flow-solver_b200/shim/stages_gpu.C" -o "$OBJ/stages_gpu.o"
g++ -o "$OUT/field_solver_stages" $STAGEOBJ "$OBJ/stages_gpu.o" $SHIMS \
    -L"$LIBDIR" -lflowgpu -Wl,-rpath,'$ORIGIN/../../flow-solver_b200/lib' -lm
echo "built $OUT/field_solver, $OUT/field_solver_gpu and $OUT/field_solver_stages"
