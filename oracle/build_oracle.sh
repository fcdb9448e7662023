#!/bin/sh
# Build the C restatement of the hot path (test infrastructure) into
# oracle/_build/libflow_oracle.so.  No FMA contraction, as in the reference.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_build"
gcc -O2 -fPIC -ffp-contract=off -std=c99 -D_DEFAULT_SOURCE -Wall -shared \
    -o "$HERE/_build/libflow_oracle.so" "$HERE/flow_oracle.c" -lm
echo "built $HERE/_build/libflow_oracle.so"
