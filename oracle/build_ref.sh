#!/usr/bin/env bash
# Builds the reference's own code, from its sources where they lie, into
# oracle/_ref/ (git-ignored; test infrastructure only, never linked by the
# product):
#   ref_mrc, ref_mrcz        the MRC class (mrc.cpp) and the MRC-gz reader
#                            (mrcz.cpp, with zlib)
#   ref_func                 func.cpp against the stand-in FFTW/libtiff headers
#                            of oracle/stubs/ (its FFT-free functions only)
#   ref_solve                mfunc.h's pair list and OD_Threshold plus the
#                            least-squares steps of DFAlign.cu:875-948, against
#                            the project's SP++ stand-in (oracle/stubs/sppp)
#   ref_pair                 cufunc.cu's pair stage and sum (cuFFT) driven by
#                            oracle/ref_pair_harness.cpp
#   dosefgpu_driftcorr_ref   the reference's whole program (dosefgpu_driftcorr.cpp,
#                            DFAlign.cu, cufunc.cu, func.cpp, mrc/mrcz/mrct.cpp,
#                            safefft.cpp) for sm_100a with cuFFT, its FFTW calls
#                            answered by cuFFT's FFTW interface (libcufftw),
#                            SP++ by oracle/stubs/sppp and libtiff by
#                            oracle/ref_tiff_stub.cpp (TIFF input unsupported)
#
# The reference tree is taken from $MC_REFERENCE_DIR (default /root/reference).
#   build_ref.sh          build what is missing or stale
#   build_ref.sh --where  print the reference's source directory; exit 1 if absent
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
SRC="${MC_REFERENCE_DIR:-/root/reference}/src-1125"
OUT="$HERE/_ref"
if [ "${1:-}" = "--where" ]; then
  if [ -f "$SRC/mrc.cpp" ]; then echo "$SRC"; exit 0; fi
  exit 1
fi
if [ ! -f "$SRC/mrc.cpp" ]; then
  echo "reference tree not present; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
stale() {  # stale <target> <inputs...>: target missing or older than an input
  local t="$1"
  shift
  [ -x "$t" ] || return 0
  local s
  for s in "$@"; do [ "$s" -nt "$t" ] && return 0; done
  return 1
}
if stale "$OUT/ref_mrc" "$HERE/ref_mrc_harness.cpp"; then
  g++ -O2 -w -I "$SRC" "$HERE/ref_mrc_harness.cpp" "$SRC/mrc.cpp" -o "$OUT/ref_mrc"
fi
if stale "$OUT/ref_mrcz" "$HERE/ref_mrcz_harness.cpp"; then
  g++ -O2 -w -I "$SRC" "$HERE/ref_mrcz_harness.cpp" "$SRC/mrc.cpp" "$SRC/mrcz.cpp" -lz -o "$OUT/ref_mrcz"
fi
if stale "$OUT/ref_func" "$HERE/ref_func_harness.cpp" "$HERE/stubs/tiffio.h"; then
  g++ -O2 -w -I "$HERE/stubs" -I "$SRC" "$HERE/ref_func_harness.cpp" "$SRC/func.cpp" "$SRC/mrc.cpp" \
      "$SRC/mrcz.cpp" -lz -lpthread -o "$OUT/ref_func"
fi
if stale "$OUT/ref_solve" "$HERE/ref_solve_harness.cpp" "$HERE/stubs/sppp/linequs2.h"; then
  g++ -O2 -w -I "$HERE/stubs/sppp" -I "$SRC" "$HERE/ref_solve_harness.cpp" -o "$OUT/ref_solve"
fi
# CUDA parts; libcuda from the toolkit's link stub, the driver's at run time
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
[ -x "$NVCC" ] || { echo "$OUT/ref_mrc"; exit 0; }
ARCH="-gencode arch=compute_100a,code=sm_100a"
CUDALIB="-L /usr/local/cuda/lib64 -L /usr/local/cuda/lib64/stubs -Wl,-rpath,/usr/local/cuda/lib64"
if stale "$OUT/ref_pair" "$HERE/ref_pair_harness.cpp" "$HERE/ref_fftw_dft.cpp"; then
  OBJ="$OUT/obj"
  mkdir -p "$OBJ"
  "$NVCC" $ARCH -O2 -w -I "$HERE/stubs" -I "$SRC" -c "$SRC/cufunc.cu" -o "$OBJ/cufunc.o"
  for s in func mrc mrcz; do
    g++ -O2 -w -I "$HERE/stubs" -I "$SRC" -I /usr/local/cuda/include -c "$SRC/$s.cpp" -o "$OBJ/$s.o"
  done
  g++ -O2 -w -I "$HERE/stubs" -c "$HERE/ref_fftw_dft.cpp" -o "$OBJ/fftw.o"
  g++ -O2 -w -I "$HERE/stubs" -I "$SRC" -I /usr/local/cuda/include -c "$HERE/ref_pair_harness.cpp" \
      -o "$OBJ/pair.o"
  g++ "$OBJ/pair.o" "$OBJ/cufunc.o" "$OBJ/func.o" "$OBJ/mrc.o" "$OBJ/mrcz.o" "$OBJ/fftw.o" \
      $CUDALIB -lcufft -lcudart -lcuda -lz -lpthread -o "$OUT/ref_pair"
fi
# the whole program, built the way its Makefile does (-O3), for sm_100a
if stale "$OUT/dosefgpu_driftcorr_ref" "$HERE/stubs/sppp/linequs2.h" "$HERE/stubs/tiffio.h" \
     "$HERE/ref_tiff_stub.cpp" "$HERE/stubs/cufftw/fftw3.h"; then
  OBJ="$OUT/obj_full"
  mkdir -p "$OBJ"
  INC="-I $HERE/stubs/cufftw -I $HERE/stubs/sppp -I $HERE/stubs -I $SRC"
  "$NVCC" $ARCH -O3 -w -Xptxas -dlcm=ca $INC -c "$SRC/DFAlign.cu" -o "$OBJ/DFAlign.o" &
  "$NVCC" $ARCH -O3 -w -Xptxas -dlcm=ca $INC -c "$SRC/cufunc.cu" -o "$OBJ/cufunc.o" &
  for s in func mrc mrcz mrct safefft dosefgpu_driftcorr; do
    g++ -O3 -w $INC -I /usr/local/cuda/include -c "$SRC/$s.cpp" -o "$OBJ/$s.o" &
  done
  g++ -O2 -w -I "$HERE/stubs" -c "$HERE/ref_tiff_stub.cpp" -o "$OBJ/tiff.o" &
  wait
  g++ "$OBJ/dosefgpu_driftcorr.o" "$OBJ/DFAlign.o" "$OBJ/cufunc.o" "$OBJ/func.o" "$OBJ/mrc.o" "$OBJ/mrcz.o" \
      "$OBJ/mrct.o" "$OBJ/safefft.o" "$OBJ/tiff.o" $CUDALIB -lcufftw -lcufft -lcudart -lcuda -lz -lpthread \
      -o "$OUT/dosefgpu_driftcorr_ref"
fi
echo "$OUT/ref_mrc"
