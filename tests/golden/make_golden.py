"""Regenerate the MRC golden fixtures with the reference's own MRC classes.

Needs oracle/_ref/ref_mrc and oracle/_ref/ref_mrcz (oracle/build_ref.sh,
reference tree present).  Writes into tests/golden/:
  ref_createMRC_17x13x2.mrc      bytes of MRC::createMRC(float*) for a known array
  stack_mode{0,1,2,6}.mrc        small stacks (written by motioncorr1exp_b200.mrc)
  ref_decode_mode{m}_f{k}.f32    MRC::read2DIm_32bit of frame k of each stack
  stack_mode{0,1,2,6}.mrc.gz     the same stacks gzip-compressed (mtime 0)
  ref_gz_decode_mode{m}_f{k}.f32 MRCZ's read2DIm_32bit of frame k (mrcz.cpp)
and, from oracle/_ref/ref_func (func.cpp's FFT-free functions):
  ref_func.json                  verifyCropSize cases, histMinMax results
  func_in_37x29.f32, ref_crop2fft_37x29.f32   crop2fft of a known image
  ref_cosmask16.c64              cosmask2d of a 16 x 16 half spectrum of ones
  func_in_400.f32, ref_dispshort_400.i16      buf2DispShort of known values
  func_in_16x9.f32, ref_moddisp_16.f32        FFTModulusToDispBuf layout
"""
import json
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
REFF = os.path.join(ROOT, "oracle", "_ref", "ref_func")

CROP_CASES = [(3838, 3710, 0, 0, 0, 1.0), (7676, 7420, 0, 0, 0, 2.0), (4096, 4096, 0, 0, 0, 1.0),
              (3838, 3710, 64, 10, 0, 1.0), (3838, 3710, 0, 0, 2048, 1.0), (3838, 3710, 3000, 0, 1000, 1.0),
              (1024, 1024, 0, 0, 0, 3.0), (1000, 999, 1, 1, 0, 1.5), (300, 292, 0, 0, 0, 2.0),
              (37, 29, 3, 2, 0, 1.0), (37, 29, 30, 2, 0, 1.0), (100, 100, 0, 0, 101, 1.0)]


def func_fixtures():
    out = {"cropsize": [], "hist": []}
    for c in CROP_CASES:
        r = subprocess.run([REFF, "cropsize"] + [str(v) for v in c], check=True, capture_output=True, text=True)
        out["cropsize"].append(list(c) + [int(r.stdout.split()[0])])
    img = (np.arange(37 * 29, dtype=np.float32) * 0.5 - 100.0).reshape(29, 37)
    img.tofile(os.path.join(HERE, "func_in_37x29.f32"))
    subprocess.run([REFF, "crop2fft", os.path.join(HERE, "func_in_37x29.f32"), "37", "29", "3", "2", "0", "1.0",
                    os.path.join(HERE, "ref_crop2fft_37x29.f32")], check=True, capture_output=True)
    subprocess.run([REFF, "cosmask", "16", os.path.join(HERE, "ref_cosmask16.c64")], check=True)
    v = np.random.default_rng(7).gamma(2.0, 3.0, 400).astype(np.float32)
    v[:3] = [1000.0, -50.0, 0.0]  # outliers beyond the clipped tails
    v.tofile(os.path.join(HERE, "func_in_400.f32"))
    for th in ("0.005", "0.02", "0.0"):
        r = subprocess.run([REFF, "hist", os.path.join(HERE, "func_in_400.f32"), "400", th], check=True,
                           capture_output=True, text=True)
        out["hist"].append([float(th)] + [float(x) for x in r.stdout.split()])
    subprocess.run([REFF, "dispshort", os.path.join(HERE, "func_in_400.f32"), "400",
                    os.path.join(HERE, "ref_dispshort_400.i16")], check=True)
    L = np.random.default_rng(8).random((16, 9)).astype(np.float32)
    L.tofile(os.path.join(HERE, "func_in_16x9.f32"))
    subprocess.run([REFF, "moddisp", os.path.join(HERE, "func_in_16x9.f32"), "16",
                    os.path.join(HERE, "ref_moddisp_16.f32")], check=True)
    with open(os.path.join(HERE, "ref_func.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


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
    if not all(os.path.exists(p) for p in (REF, REFZ, REFF)):
        sys.exit("oracle/_ref/ref_mrc, ref_mrcz or ref_func missing: run oracle/build_ref.sh")
    func_fixtures()
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
