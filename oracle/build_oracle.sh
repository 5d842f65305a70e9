#!/bin/bash
# ORACLE recipe — test infrastructure only.  Builds the CPU restatement
# (hpgl_oracle.cpp + textio_oracle.cpp + variogram_oracle.cpp + lapack_restated.c) into oracle/_build/libhpgl_oracle.so.
# Needs only gcc/g++ with OpenMP, so it also builds on the GPU machine.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_build
mkdir -p "$OUT"
gcc -O2 -ffp-contract=off -fPIC -c "$HERE/lapack_restated.c" -o "$OUT/lapack_restated.o"
g++ -std=gnu++17 -O2 -ffp-contract=off -fopenmp -fPIC -c "$HERE/hpgl_oracle.cpp" -o "$OUT/hpgl_oracle.o"
g++ -std=gnu++17 -O2 -fPIC -c "$HERE/textio_oracle.cpp" -o "$OUT/textio_oracle.o"
g++ -std=gnu++17 -O2 -ffp-contract=off -fPIC -c "$HERE/variogram_oracle.cpp" -o "$OUT/variogram_oracle.o"
g++ -shared -fopenmp -o "$OUT/libhpgl_oracle.so.tmp" "$OUT/hpgl_oracle.o" "$OUT/textio_oracle.o" \
    "$OUT/variogram_oracle.o" "$OUT/lapack_restated.o"
mv "$OUT/libhpgl_oracle.so.tmp" "$OUT/libhpgl_oracle.so"
echo "built $OUT/libhpgl_oracle.so"
