#!/usr/bin/env bash
# Builds the parts of the reference that compile from their own sources into
# oracle/_ref/ (git-ignored): the MRC class (mrc.cpp), the MRC-gz reader on
# top of it (mrcz.cpp, with zlib), and func.cpp against the stand-in FFTW and
# libtiff headers of oracle/stubs/ (only its FFT-free functions are called).
# The alignment code needs FFTW3, SP++ 3.0 and libtiff, which are not
# installed, so it is not built here.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
SRC=/root/reference/src-1125
OUT="$HERE/_ref"
if [ ! -f "$SRC/mrc.cpp" ]; then
  echo "reference tree not present; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
if [ ! -x "$OUT/ref_mrc" ] || [ "$HERE/ref_mrc_harness.cpp" -nt "$OUT/ref_mrc" ]; then
  g++ -O2 -w -I "$SRC" "$HERE/ref_mrc_harness.cpp" "$SRC/mrc.cpp" -o "$OUT/ref_mrc"
fi
if [ ! -x "$OUT/ref_mrcz" ] || [ "$HERE/ref_mrcz_harness.cpp" -nt "$OUT/ref_mrcz" ]; then
  g++ -O2 -w -I "$SRC" "$HERE/ref_mrcz_harness.cpp" "$SRC/mrc.cpp" "$SRC/mrcz.cpp" -lz -o "$OUT/ref_mrcz"
fi
if [ ! -x "$OUT/ref_func" ] || [ "$HERE/ref_func_harness.cpp" -nt "$OUT/ref_func" ]; then
  g++ -O2 -w -I "$HERE/stubs" -I "$SRC" "$HERE/ref_func_harness.cpp" "$SRC/func.cpp" "$SRC/mrc.cpp" \
      "$SRC/mrcz.cpp" -lz -lpthread -o "$OUT/ref_func"
fi
# the reference's pair stage (cufunc.cu with cuFFT; FFTW's calls answered by
# the direct DFTs of ref_fftw_dft.cpp); libcuda from the toolkit's link stub,
# the driver's at run time
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
if [ -x "$NVCC" ] && { [ ! -x "$OUT/ref_pair" ] || [ "$HERE/ref_pair_harness.cpp" -nt "$OUT/ref_pair" ] \
     || [ "$HERE/ref_fftw_dft.cpp" -nt "$OUT/ref_pair" ]; }; then
  OBJ="$OUT/obj"
  mkdir -p "$OBJ"
  "$NVCC" -gencode arch=compute_100a,code=sm_100a -O2 -w -I "$HERE/stubs" -I "$SRC" -c "$SRC/cufunc.cu" \
      -o "$OBJ/cufunc.o"
  for s in func mrc mrcz; do
    g++ -O2 -w -I "$HERE/stubs" -I "$SRC" -I /usr/local/cuda/include -c "$SRC/$s.cpp" -o "$OBJ/$s.o"
  done
  g++ -O2 -w -I "$HERE/stubs" -c "$HERE/ref_fftw_dft.cpp" -o "$OBJ/fftw.o"
  g++ -O2 -w -I "$HERE/stubs" -I "$SRC" -I /usr/local/cuda/include -c "$HERE/ref_pair_harness.cpp" \
      -o "$OBJ/pair.o"
  g++ "$OBJ/pair.o" "$OBJ/cufunc.o" "$OBJ/func.o" "$OBJ/mrc.o" "$OBJ/mrcz.o" "$OBJ/fftw.o" \
      -L /usr/local/cuda/lib64 -L /usr/local/cuda/lib64/stubs -Wl,-rpath,/usr/local/cuda/lib64 \
      -lcufft -lcudart -lcuda -lz -lpthread -o "$OUT/ref_pair"
fi
echo "$OUT/ref_mrc"
