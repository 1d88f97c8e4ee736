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
and, from oracle/_ref/ref_solve (mfunc.h + the steps of DFAlign.cu:875-948
against the project's SP++ stand-in):
  ref_solve_cases.json           pair shifts in, pair list, ki1, kept rows, ki2
                                 and per-step shifts out, for SOLVE_CASES
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
REFS = os.path.join(ROOT, "oracle", "_ref", "ref_solve")

# (nframe, fod, kithresh, noise px, outliers, seed): exact systems, noisy ones,
# planted outliers, thresholds that keep only a rank-deficient prefix (the
# rank loop must add rows), the benchmark shapes (16/2, 40/7, 50/2, 60/2)
SOLVE_CASES = [(6, 0, 1.0, 0.0, 0, 1), (12, 2, 1.0, 0.05, 2, 2), (12, 2, 0.01, 0.3, 0, 3),
               (16, 2, 1.0, 0.1, 1, 4), (16, 2, 0.001, 0.5, 3, 5), (40, 7, 1.0, 0.2, 4, 6),
               (40, 7, 0.05, 0.2, 0, 7), (50, 2, 1.0, 0.3, 5, 8), (60, 2, 0.2, 0.4, 6, 9),
               (9, 4, 0.5, 1.0, 2, 10), (20, 9, 0.0, 0.1, 0, 11)]


def run_ref_solve(nframe, fod, kithresh, b):
    """Runs oracle/_ref/ref_solve; returns its outputs as a dict."""
    inp = f"{nframe} {fod} {kithresh!r}\n" + "".join(f"{float(x.real)!r} {float(x.imag)!r}\n" for x in b)
    out = subprocess.run([REFS], input=inp, check=True, capture_output=True, text=True).stdout.split("\n")
    k = 0
    res = {}
    np_ = int(out[k].split()[1])
    res["pairs"] = [[int(v) for v in out[k + 1 + i].split()] for i in range(np_)]
    k += 1 + np_
    assert out[k] == "ki1"
    res["ki1"] = [float(v) for v in out[k + 1:k + 1 + np_]]
    k += 1 + np_
    ng = int(out[k].split()[1])
    res["good"] = [int(v) for v in out[k + 1:k + 1 + ng]]
    k += 1 + ng
    assert out[k] == "ki2"
    res["ki2"] = [float(v) for v in out[k + 1:k + 1 + ng]]
    k += 1 + ng
    assert out[k] == "shift"
    res["shift"] = [[float(v) for v in out[k + 1 + i].split()] for i in range(nframe - 1)]
    return res


def solve_case_input(nframe, fod, noise, outliers, seed):
    """Pair shifts of a random drift: float32-rounded like the pair stage's."""
    rng = np.random.default_rng(seed)
    dist = max(1, min(nframe // 2 - fod, nframe // 2))
    pairs = [(i, j) for i in range(nframe) for j in range(i + dist, nframe)]
    steps = rng.normal(0, 1, nframe - 1) + 1j * rng.normal(0, 1, nframe - 1)
    b = np.array([steps[i:j].sum() for i, j in pairs])
    b += noise * (rng.normal(size=len(pairs)) + 1j * rng.normal(size=len(pairs)))
    for r in rng.choice(len(pairs), size=outliers, replace=False):
        b[r] += rng.choice([-1, 1]) * rng.uniform(3, 8) + 1j * rng.uniform(-5, 5)
    return (b.real.astype(np.float32) + 1j * b.imag.astype(np.float32)).astype(np.complex128)


def solve_fixtures():
    cases = []
    for nf, fod, kit, noise, nout, seed in SOLVE_CASES:
        b = solve_case_input(nf, fod, noise, nout, seed)
        r = run_ref_solve(nf, fod, kit, b)
        r.update({"nframe": nf, "fod": fod, "kithresh": kit,
                  "b": [[float(x.real), float(x.imag)] for x in b]})
        cases.append(r)
    with open(os.path.join(HERE, "ref_solve_cases.json"), "w") as f:
        json.dump(cases, f)
        f.write("\n")

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
    if not all(os.path.exists(p) for p in (REF, REFZ, REFF, REFS)):
        sys.exit("oracle/_ref/ref_mrc, ref_mrcz, ref_func or ref_solve missing: run oracle/build_ref.sh")
    if sys.argv[1:] == ["solve"]:
        solve_fixtures()
        return
    func_fixtures()
    solve_fixtures()
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
