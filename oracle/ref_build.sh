#!/usr/bin/env bash
# Compiles the reference engine for the oracle-pinning build:
#   $MS_REFERENCE_DIR/GUI Simulation/UnmanagedGUISimulation.cu  (unchanged;
#   MS_REFERENCE_DIR defaults to the read-only checkout of the build machine,
#   and the build is skipped where no reference sources are found)
#   + oracle/ref_shim (empty Stdafx.h and Boost stand-ins, and the
#     cudaMemcpyToSymbol string-name fix, force-included)
#   + oracle/ref_driver.cpp (C entry points for the golden-vector generator;
#     it includes the reference source file, so both form one translation unit)
# into oracle/_ref/libmsref.so.  Nothing from the reference tree is copied.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${MS_REFERENCE_DIR:-/root/reference}/GUI Simulation"
OUT="$HERE/_ref"
if [ ! -f "$REF/UnmanagedGUISimulation.cu" ]; then
  echo "reference sources not found under $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC="${NVCC:-nvcc}"
ARCH="-gencode arch=compute_100a,code=sm_100a"
COMMON="-std=c++14 -O2 -Xcompiler -fPIC -w -I$HERE/ref_shim"
if [ "$OUT/libmsref.so" -nt "$REF/UnmanagedGUISimulation.cu" ] && [ "$OUT/libmsref.so" -nt "$HERE/ref_driver.cpp" ] \
   && [ "$OUT/libmsref.so" -nt "$HERE/ref_shim/ref_symbol_fix.h" ]; then
  exit 0
fi
$NVCC $ARCH $COMMON -I"$REF" -include cfloat -include "$HERE/ref_shim/ref_symbol_fix.h" \
  -x cu -c "$HERE/ref_driver.cpp" -o "$OUT/ref_driver.o"
$NVCC $ARCH -shared -o "$OUT/libmsref.so" "$OUT/ref_driver.o" -lcufft -lcublas \
  -Xlinker -rpath,/usr/local/cuda/lib64
echo "$OUT/libmsref.so"
