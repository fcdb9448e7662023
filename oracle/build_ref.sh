#!/bin/sh
# Build the oracle's copy of the reference solver: the reference's own *.C
# files, compiled where they lie (read-only) with the flags of its Makefile
# (Makefile:19: -Wno-deprecated -Wall -ansi -pedantic -O3), plus
#   - shims/gsl_shim.c, shims/lapack_shim.c: stand-ins for GSL qags and
#     LAPACK dgesvd_ (neither library is part of the reference tree),
#   - ref_harness.cpp: C entry points replacing main.C's driver loop.
# Output: oracle/_ref/libflowref.so (git-ignored; travels with the tree).
# Usage: sh oracle/build_ref.sh reference_dir   (or FLOW_REFERENCE_DIR=... sh oracle/build_ref.sh)
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-$FLOW_REFERENCE_DIR}
if [ -z "$REF" ]; then
  echo "build_ref.sh: give the reference directory as the argument or in FLOW_REFERENCE_DIR" >&2
  exit 1
fi
OUT="$HERE/_ref"
HOST="$HERE/../flow-solver_b200/csrc/host"
if [ ! -f "$REF/solve.C" ]; then
  echo "build_ref.sh: reference sources not found at $REF" >&2
  exit 1
fi
mkdir -p "$OUT/obj"
CFLAGS="-Wno-deprecated -Wall -ansi -pedantic -O3 -fPIC"
INC="-I$REF/include -I$HERE/shims -I$HOST"
for f in "$REF"/*.C; do
  b=$(basename "$f" .C)
  [ "$b" = main ] && continue
  g++ -x c++ $CFLAGS $INC -w -c "$f" -o "$OUT/obj/$b.o"
done
gcc -O2 -fPIC -I"$HOST" -c "$HOST/quadrature.c" -o "$OUT/obj/quadrature.o"
gcc -O2 -fPIC -I"$HOST" -c "$HOST/svd.c" -o "$OUT/obj/svd.o"
gcc -O2 -fPIC -I"$HERE/shims" -I"$HOST" -c "$HERE/shims/gsl_shim.c" -o "$OUT/obj/gsl_shim.o"
gcc -O2 -fPIC -I"$HOST" -c "$HERE/shims/lapack_shim.c" -o "$OUT/obj/lapack_shim.o"
g++ -O2 -fPIC -Wall $INC -c "$HERE/ref_harness.cpp" -o "$OUT/obj/ref_harness.o"
g++ -shared -o "$OUT/libflowref.so" "$OUT"/obj/*.o -lm
echo "built $OUT/libflowref.so"
