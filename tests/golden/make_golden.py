"""Regenerate the MRC golden fixtures with the reference's own MRC classes.

Needs oracle/_ref/ref_mrc and oracle/_ref/ref_mrcz (oracle/build_ref.sh,
reference tree present).  Writes into tests/golden/:
  ref_createMRC_17x13x2.mrc      bytes of MRC::createMRC(float*) for a known array
  stack_mode{0,1,2,6}.mrc        small stacks (written by motioncorr1exp_b200.mrc)
  ref_decode_mode{m}_f{k}.f32    MRC::read2DIm_32bit of frame k of each stack
  stack_mode{0,1,2,6}.mrc.gz     the same stacks gzip-compressed (mtime 0)
  ref_gz_decode_mode{m}_f{k}.f32 MRCZ's read2DIm_32bit of frame k (mrcz.cpp)
"""
import gzip
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from motioncorr1exp_b200 import mrc  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "ref_mrc")
REFZ = os.path.join(ROOT, "oracle", "_ref", "ref_mrcz")


def image_array():
    x = np.arange(17 * 13 * 2, dtype=np.float64).reshape(2, 13, 17)
    return (np.sin(x * 0.37) * 1000.0 + x * 0.125).astype(np.float32)


def stack_array(mode):
    rng = np.random.default_rng(100 + mode)
    if mode == 0:
        return rng.integers(0, 256, (3, 11, 9)).astype(np.uint8)    # includes >= 128
    if mode == 1:
        return rng.integers(-32768, 32767, (3, 11, 9)).astype(np.int16)
    if mode == 6:
        return rng.integers(0, 65535, (3, 11, 9)).astype(np.uint16)
    return rng.normal(0, 100, (3, 11, 9)).astype(np.float32)


def main():
    if not os.path.exists(REF) or not os.path.exists(REFZ):
        sys.exit("oracle/_ref/ref_mrc or ref_mrcz missing: run oracle/build_ref.sh")
    img = image_array()
    tmp = os.path.join(HERE, "_in.f32")
    img.tofile(tmp)
    subprocess.run([REF, "write", os.path.join(HERE, "ref_createMRC_17x13x2.mrc"), "17", "13", "2", tmp], check=True)
    os.remove(tmp)
    for mode in (0, 1, 2, 6):
        path = os.path.join(HERE, f"stack_mode{mode}.mrc")
        mrc.write_stack(path, stack_array(mode), mode)
        for k in range(3):
            subprocess.run([REF, "read", path, str(k), os.path.join(HERE, f"ref_decode_mode{mode}_f{k}.f32")],
                           check=True)
        gz = path + ".gz"
        with open(path, "rb") as f, open(gz, "wb") as g:
            g.write(gzip.compress(f.read(), mtime=0))
        for k in (2, 0, 1):  # a backward seek after the first read
            subprocess.run([REFZ, "read", gz, str(k), os.path.join(HERE, f"ref_gz_decode_mode{mode}_f{k}.f32")],
                           check=True)


if __name__ == "__main__":
    main()
