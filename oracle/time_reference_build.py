"""Times the reference's own program (cuFFT build) against this path's CLI on
the benchmark movie, and compares their results.

TEST INFRASTRUCTURE: runs oracle/_ref/dosefgpu_driftcorr_ref, the
reference's dosefgpu_driftcorr built from its sources by oracle/build_ref.sh
(SP++, FFTW and libtiff answered by project stand-ins: oracle/stubs/sppp,
cuFFT's FFTW interface, oracle/ref_tiff_stub.cpp).

Workload: the 40-frame 3838x3710 uint8 movie (mean 1.2 e/px/frame, seeded
random-walk + linear drift from motioncorr1exp_b200.synth.make_movie_torch),
written as an MRC (mode 0) to /dev/shm; both programs run it with
-fod 7 -bft 150 -pbx 96 -atm 1 -dsp 0 and write the corrected sum (-fcs) and
the log (-flg).  Each timing is the wall clock of the whole process (MRC
read, CUDA context, alignment, sum, MRC write), one warm-up run first.

  python oracle/time_reference_build.py [--runs R] [--frames F] [--out result.json]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

REF = os.path.join(ROOT, "oracle", "_ref", "dosefgpu_driftcorr_ref")
CLI = os.path.join(ROOT, "motioncorr1exp_b200", "lib", "dosefgpu_driftcorr")
FLAGS = ["-fod", "7", "-bft", "150", "-pbx", "96", "-atm", "1", "-dsp", "0"]


def run(exe, stack, tag, d):
    log = os.path.join(d, f"{tag}.log")
    fcs = os.path.join(d, f"{tag}_sum.mrc")
    if os.path.exists(log):
        os.remove(log)
    t0 = time.perf_counter()
    r = subprocess.run([exe, stack, "-fcs", fcs, "-flg", log] + FLAGS, cwd=d, capture_output=True, text=True,
                       timeout=1800)
    t = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"{tag}: rc {r.returncode}: {r.stdout[-1000:]} {r.stderr[-1000:]}")
    return t, log, fcs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=3)
    ap.add_argument("--frames", type=int, default=40)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default="")
    a = ap.parse_args()
    import torch
    from motioncorr1exp_b200 import mrc, synth
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_gpu_reference_full import parse_log

    frames, truth = synth.make_movie_torch(3838, 3710, a.frames, mean=1.2, seed=a.seed, dtype="u8", kind="linear",
                                           speed=0.3, rw_sigma=0.5, device="cuda")
    host = frames.cpu().numpy()
    del frames
    torch.cuda.empty_cache()
    base = "/dev/shm" if os.path.isdir("/dev/shm") else None
    with tempfile.TemporaryDirectory(dir=base) as d:
        stack = os.path.join(d, "c2.mrc")
        mrc.write_stack(stack, host, 0)
        res = {}
        for tag, exe in (("reference", REF), ("ours", CLI)):
            run(exe, stack, tag, d)  # warm-up (page cache, driver)
            ts = []
            for _ in range(a.runs):
                t, log, fcs = run(exe, stack, tag, d)
                ts.append(t)
            res[tag] = {"wall_s": ts, "median_s": statistics.median(ts),
                        "frames_per_s": a.frames / statistics.median(ts),
                        "log": parse_log(open(log).read()),
                        "image": mrc.read_stack(fcs)[0][0].astype(np.float64)}
    r, o = res["reference"], res["ours"]
    rs = np.array([(q[2], q[3]) for q in r["log"]["pairs"]])
    os_ = np.array([(q[2], q[3]) for q in o["log"]["pairs"]])
    fr, fo = np.array(r["log"]["shift"]), np.array(o["log"]["shift"])
    out = {
        "workload": f"{a.frames} frames 3838x3710 uint8 (MRC mode 0), mean 1.2 e/px/frame, seed {a.seed}; "
                    + " ".join(FLAGS),
        "timing": "wall clock of the whole process per movie (MRC read from /dev/shm, CUDA context, alignment, "
                  "sum, MRC write), median of the runs after one warm-up",
        "reference_build": "oracle/_ref/dosefgpu_driftcorr_ref: the reference's sources, -O3, sm_100a, cuFFT; "
                           "FFTW via libcufftw, SP++ via oracle/stubs/sppp",
        "reference_wall_s": r["wall_s"], "ours_cli_wall_s": o["wall_s"],
        "reference_frames_per_s": r["frames_per_s"], "ours_cli_frames_per_s": o["frames_per_s"],
        "cli_speedup": r["median_s"] / o["median_s"],
        "pairs": len(rs), "pair_shift_lines_differing": int(np.sum(np.any(np.abs(rs - os_) > 1e-6, axis=1))),
        "frame_shift_max_diff_px": float(np.max(np.abs(fr - fo))),
        "sum_rel_l2_ours_vs_reference": float(np.linalg.norm(o["image"] - r["image"]) / np.linalg.norm(r["image"])),
    }
    line = json.dumps(out)
    print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
