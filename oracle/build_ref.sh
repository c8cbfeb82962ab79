#!/usr/bin/env bash
# Builds the reference's own CUDA path (FD2DGPU.cu + born.cu, compiled where they lie in the
# reference tree) plus oracle/ref_harness.cu, and its CPU acoustic stepper (main.cpp +
# laplace.cpp, through oracle/ref_cpu.cpp), into oracle/_ref/libds2dref.so.  Test
# infrastructure only: the library is the parity checker, never the product.  Flags follow the
# reference Makefile (nvcc -O3 -w -DELASTIC -DORDER=12) with an explicit sm_100a target.
#
#   oracle/build_ref.sh [--if-present]
#
# The reference tree is read from $DS2D_REFERENCE, default /root/reference.  With --if-present a
# missing tree is not an error (nothing is built), so build steps can call the recipe anywhere.
set -euo pipefail
REF="${DS2D_REFERENCE:-/root/reference}"
if [ ! -f "$REF/FD2DGPU.cu" ]; then
  if [ "${1:-}" = "--if-present" ]; then
    echo "reference tree not found at $REF: oracle/_ref not built"
    exit 0
  fi
  echo "reference tree not found at $REF (set DS2D_REFERENCE)" >&2
  exit 1
fi
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
mkdir -p "$OUT"
FLAGS="-O3 -w -DELASTIC -DORDER=12 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC"
nvcc $FLAGS -I"$REF" -c "$REF/born.cu" -o "$OUT/born.o"
nvcc $FLAGS -I"$REF" -c "$HERE/ref_harness.cu" -o "$OUT/ref_harness.o"
# main.cpp (its CPU acoustic stepper) and laplace.cpp, compiled as the reference's Makefile does
# (g++ -O3 -w -fopenmp -DELASTIC), main.cpp against the project's stub mpi.h
CXXF="-O3 -w -fopenmp -fPIC -DELASTIC -I$REF -I$HERE/stub -I${CUDA_HOME:-/usr/local/cuda}/include"
g++ $CXXF -c "$REF/laplace.cpp" -o "$OUT/laplace.o"
g++ $CXXF -c "$HERE/ref_cpu.cpp" -o "$OUT/ref_cpu.o"
nvcc -shared -gencode arch=compute_100a,code=sm_100a -o "$OUT/libds2dref.so" \
  "$OUT/ref_harness.o" "$OUT/born.o" "$OUT/laplace.o" "$OUT/ref_cpu.o" -lcublas -lcufft -lgomp
rm -f "$OUT/born.o" "$OUT/ref_harness.o" "$OUT/laplace.o" "$OUT/ref_cpu.o"
echo "built $OUT/libds2dref.so"
