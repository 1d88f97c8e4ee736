#!/usr/bin/env python
"""Aligned frames/s of the drift-correction path on the 3838x3710x40 uint8 movie.

Workload (one "step" = one whole movie through the path): 40 frames of
3838x3710 uint8 Poisson counts (mean 1.2 e/px/frame), seeded synthetic
signal, random-walk + linear drift; -fod 7 -bft 150 -pbx 96 -atm 1 -bin 1
(square crop 3710, 378 frame pairs).  Inputs are larger than L2 (570 MB raw
frames, 2.2 GB of spectra), so no flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: one process per GPU, each aligning its own movie (replicas; the
path has no exchange step), max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "aligned frames/s at 3838x3710x40"
UNIT = "frames/s"
WORKLOAD = ("c2: 40 frames 3838x3710 uint8 (MRC mode 0), mean 1.2 e/px/frame, RW 0.5 + 0.3 px/frame drift; "
            "-bin 1 -fod 7 -bft 150 -pbx 96 -atm 1 -itr 0; crop 3710^2, 378 pairs")
FALLBACK_HBM_GBS = 6650.0


def c2_params(api):
    return api.Params(bin=1.0, FrameDistOffset=7, bfactor=150.0, CCPeakSearchDim=96, bAlignToMid=1,
                      NoisePeakSize=0, kiThresh=1.0)


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(kernel):
    """bytes per launch from the committed ncu summary (profiles/traffic.txt)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and parts[0] == kernel and parts[1] == "c2":
                    return float(parts[2])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- CPU arms --
def oracle_sample(seed=0, n_pairs=1):
    """Time the FP64 oracle on a bounded sample of the workload: the forward
    transform of one frame, ``n_pairs`` pair correlations + sub-pixel peaks and
    one frame of the phase-shift sum, scaled to frames/s with P/F = 378/40."""
    import numpy as np
    from motioncorr1exp_b200 import synth
    from oracle import mc_oracle as O
    mv, _ = synth.make_workload("c2", seed=seed, nframes=2)
    nu = O.verify_crop_size(3838, 3710, 0, 0, 0, 1.0)
    t0 = time.perf_counter()
    F0 = O.forward_spectrum(O.decode_frame(mv.frames[0], 0), 0, 0, nu, nu)
    t1 = time.perf_counter()
    F1 = O.forward_spectrum(O.decode_frame(mv.frames[1], 0), 0, 0, nu, nu)
    mask = O.bfactor_mask(nu, 150.0)
    t2 = time.perf_counter()
    for _ in range(n_pairs):
        O.find_shift(O.cc_box(O.cc_map(F0, F1, mask, nu), nu, 96), nu, 0)
    t3 = time.perf_counter()
    S = O.phase_shift(F0, 0.3, -0.2) + F1
    t4 = time.perf_counter()
    O.spectrum_to_image(S)            # once per movie: amortised over its 40 frames
    t5 = time.perf_counter()
    t_fwd = t1 - t0
    t_pair = (t3 - t2) / n_pairs
    t_sum = (t4 - t3) + (t5 - t4) / 40.0
    per_frame = t_fwd + (378.0 / 40.0) * t_pair + t_sum
    return 1.0 / per_frame, {"fwd_s": t_fwd, "pair_s": t_pair, "sum_s": t_sum}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        v, parts = oracle_sample(seed=args.seed, n_pairs=1)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    sample = ("per step: FP64 oracle (numpy/scipy pocketfft, all host threads) on one 3710^2 frame forward "
              "R2C, one pair cross-correlation + FindShift, one frame phase-shift; scaled by P/F = 378/40 "
              "to frames/s")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * 40 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU arm --
def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    from motioncorr1exp_b200 import api, synth

    from motioncorr1exp_b200 import dist as D
    rank, world, local = D.world()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()

    nx, ny, nz = 3838, 3710, args.frames
    frames, truth = synth.make_movie_torch(nx, ny, nz, mean=1.2, seed=args.seed + rank, dtype="u8",
                                           kind="linear", speed=0.3, rw_sigma=0.5, device=f"cuda:{local}")
    host = torch.empty(frames.shape, dtype=torch.uint8, pin_memory=True)
    host.copy_(frames)
    p = c2_params(api)
    p.GPUNum = local
    p = api.verify_params(p, nz)
    plan = api.Plan(p, nx, ny, nz, 0)
    stream = torch.cuda.ExternalStream(plan.stream, device=f"cuda:{local}")
    image = torch.empty((plan.nsam, plan.nsam), dtype=torch.float32, pin_memory=True)
    image_np = image.numpy()

    def step_resident():
        plan.run(want_image=False)

    host_np = host.numpy()

    def step_e2e():
        # pinned H2D overlapped with the forward transforms, image D2H into pinned memory
        plan.run_host(host_np, out=image_np)

    plan.load_frames_device(frames.data_ptr(), 0, nz)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step_resident()

    # ---- device-resident timed region
    plan.reset_stats()
    plan.set_profiling(True)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step_resident()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    plan.set_profiling(False)
    ms = e0.elapsed_time(e1)
    stats = plan.kernel_stats()
    shifts = plan.frame_shifts()
    ms_max = D.max_over_ranks(ms)

    # ---- end-to-end through the public API from pinned host buffers
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        step_e2e()
    f1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = D.max_over_ranks(f0.elapsed_time(f1))

    truth_rmse = float(np.sqrt(np.mean(np.sum((shifts + (truth - truth[0])) ** 2, axis=1))))

    if rank == 0:
        value = nz * args.steps * world / (ms_max / 1000.0)
        e2e_value = nz * args.steps * world / (e2e_ms / 1000.0)
        dom = max(stats, key=lambda k: stats[k]["ms"])
        d = stats[dom]
        per_launch_ms = d["ms"] / max(d["launches"], 1)
        per_launch_bytes = d["bytes"] / max(d["launches"], 1)
        peak, peak_kind = measured_peak()
        achieved = per_launch_bytes / (per_launch_ms / 1000.0) / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": committed_traffic(dom), "peak_source": peak_kind,
                "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms}
        launches = int(sum(v["launches"] for v in stats.values()))
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD if nz == 40 else f"profiling case: {nz} frames, else as c2",
                           "nsam": plan.nsam, "pairs": plan.npairs,
                           "l2": "inputs larger than L2 (570 MB frames, 2.2 GB spectra per movie), no flush",
                           "parallelism": f"replicas x{world}"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(host.numel()),
                        "d2h_bytes_per_step": int(image.numel() * 4)},
                "gpu_launches": launches, "roofline": roof,
                "kernels": {k: {"ms_per_step": v["ms"] / args.steps, "launches": v["launches"],
                                "GBps": (v["bytes"] / (v["ms"] / 1000.0) / 1e9) if v["ms"] > 0 else None}
                            for k, v in stats.items()},
                "shift_rmse_vs_truth_px": truth_rmse,
                "clocks": clk.summary()}
        if world == 1 and not args.no_cpu_baseline:
            v, parts = oracle_sample(seed=args.seed)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": "FP64 oracle, one frame forward + one pair + one frame sum at "
                                              "3710^2, scaled by P/F = 378/40; " +
                                              ", ".join(f"{k}={x:.2f}" for k, x in parts.items())}
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--frames", type=int, default=40,
                    help="movie length; 40 is the benchmark workload, fewer only for profiling captures")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
