#!/usr/bin/env bash
# Builds the parts of the reference that compile from their own sources into
# oracle/_ref/ (git-ignored): the MRC class (mrc.cpp) and the MRC-gz reader
# on top of it (mrcz.cpp, with zlib).  The alignment code needs FFTW3, SP++
# 3.0 and libtiff, which are not installed, so it is not built here.
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
echo "$OUT/ref_mrc"
