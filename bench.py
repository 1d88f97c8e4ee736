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
WORKLOADS_TEXT = {
    "c1": "c1: 16 frames 1024x1024 float32 (MRC mode 2), mean 1.5 e/px/frame, 0.4 px/frame linear + RW 0.3; "
          "-bin 1 -fod 2 -bft 150 -pbx 96 -nps 0; 55 pairs",
    "c3": "c3: 50 frames 7676x7420 uint8, mean 0.3 e/px/frame, RW 0.5 + 0.3 px/frame; -bin 2 (crop 7420, "
          "Fourier crop to 3710), -fod 2; 378 pairs",
    "c4": "c4: 60 frames 4096x4096 float32, mean 1.0 e/px/frame, RW 0.8 + sinusoid 1.5 px period 20; -fod 2, "
          "-itr 3 -ith 0.01, gradient refinement (-ref 1); 528 pairs",
}


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
    """nvidia-smi clocks and throttle reasons during the timed region.

    The sampler starts before the region and waits for its first sample (the
    tool takes a moment to start); samples are stamped on arrival and only
    those inside the region count (the first one after its start when the
    region is shorter than the sampling period)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period_ms=20):
        self.index = index
        self.period_ms = period_ms
        self.proc = None
        self.samples = []       # (host time, line)
        self.t0 = self.t1 = None

    def _reader(self):
        for line in self.proc.stdout:
            if line.strip():
                self.samples.append((time.perf_counter(), line))

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._reader, daemon=True)
            self.thread.start()
            deadline = time.perf_counter() + 10.0
            while not self.samples and time.perf_counter() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *exc):
        self.t1 = time.perf_counter()
        if self.proc:
            time.sleep(2.0 * self.period_ms / 1000.0)   # one more sample after the region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self):
        inside = [l for t, l in self.samples if self.t0 <= t <= self.t1]
        if not inside:
            inside = [l for t, l in self.samples if t >= self.t0][:1]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in inside:
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

    w = dict(synth.WORKLOADS[args.workload])
    flags = dict(w.pop("flags"))
    if args.workload == "c4":
        flags["refine"] = 1            # the gradient refinement after the iterations
    nx, ny = w["nx"], w["ny"]
    nz = args.frames or w["nframes"]
    mode = 0 if w["dtype"] == "u8" else 2
    frames, truth = synth.make_movie_torch(nx, ny, nz, mean=w["mean"], seed=args.seed + rank, dtype=w["dtype"],
                                           kind=w["kind"], speed=w.get("speed", 0.4),
                                           rw_sigma=w.get("rw_sigma", 0.3), amp=w.get("amp", 1.5),
                                           period=w.get("period", 20.0), device=f"cuda:{local}")
    host = torch.empty(frames.shape, dtype=frames.dtype, pin_memory=True)
    host.copy_(frames)
    p = c2_params(api) if args.workload == "c2" else api.Params(**flags)
    p.GPUNum = local
    p = api.verify_params(p, nz)
    plan = api.Plan(p, nx, ny, nz, mode)
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

    def timed(fn):
        barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        out = fn()
        t1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return D.max_over_ranks(t0.elapsed_time(t1)), out

    # ---- single plan, device-resident frames: the movie graph replayed per step
    plan.reset_stats()
    single_ms, _ = timed(lambda: [step_resident() for _ in range(args.steps)])
    launches_per_movie = sum(v["launches"] for v in plan.kernel_stats().values()) / args.steps
    shifts = plan.frame_shifts()

    # ---- headline: the batch API (--lanes lanes, each its own stream, plan and
    # graph) over K movies whose frames are resident in HBM; the lanes overlap
    # one movie's serial tail (peak search, solve, sum) with the next one's
    # transforms
    batch = api.Batch(local, args.lanes)
    dev = [{"params": p, "nx": nx, "ny": ny, "nz": nz, "mode": mode, "device_ptr": frames.data_ptr()}
           for _ in range(args.steps)]
    for _ in range(max(1, args.warmup // 2)):
        batch.run(dev[:2])
    with ClockSampler(local) as clk:
        ms_max, res_dev = timed(lambda: batch.run(dev))
    dev_lat = [r["end_ms"] - r["start_ms"] for r in res_dev]
    launches = int(round(launches_per_movie * args.steps))

    # ---- per-kernel CUDA-event durations: a profiled pass of the single plan
    # (events around every launch, so no graph), for the roofline
    plan.reset_stats()
    plan.set_profiling(True)
    prof_steps = min(args.steps, 3)
    for _ in range(prof_steps):
        step_resident()
    torch.cuda.synchronize()
    plan.set_profiling(False)
    stats = plan.kernel_stats()

    # ---- end-to-end through the same batch API from pinned host buffers:
    # every step uploads its movie and reads its image back
    images = [torch.empty((plan.nsam, plan.nsam), dtype=torch.float32, pin_memory=True).numpy()
              for _ in range(args.steps)]
    mv = [{"params": p, "nx": nx, "ny": ny, "nz": nz, "mode": mode, "frames": host_np, "image": im}
          for im in images]
    batch.run(mv[:2])
    e2e_ms, res = timed(lambda: batch.run(mv))
    e2e_lat = [r["end_ms"] - r["start_ms"] for r in res]
    batch.close()
    # the single-plan form of the same call, one movie at a time
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    single_e2e_ms, _ = timed(lambda: [step_e2e() for _ in range(args.steps)])

    # shifts come in binned pixels (nsam / nsam_unbin of a raw pixel)
    to_binned = plan.nsam / plan.info["nsam_unbin"]
    truth_rmse = float(np.sqrt(np.mean(np.sum((shifts + to_binned * (truth - truth[0])) ** 2, axis=1))))

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
                "frac": achieved / peak, "traffic": committed_traffic(dom) if args.workload == "c2" else None,
                "peak_source": peak_kind, "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms}
        if dom == "k_pair_cols":
            # the kernel is FP32-issue bound: its compute roofline beside the
            # HBM one.  Algorithmic FLOPs per (pair, column): the cross power
            # x B-factor (8 n), P inverse FFTs of length Q (5 Q log2 Q each,
            # the usual FFT count) and the 96-row P-term sums (8 P box)
            info = plan.info
            n, P, Q = plan.nsam, info["prune_p"], info["prune_q"]
            per_pc = 8.0 * n + P * 5.0 * Q * np.log2(Q) + 8.0 * P * p.CCPeakSearchDim
            flops = per_pc * plan.npairs * (n // 2 + 1)
            fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
            roof["fp32"] = {"achieved": flops / (per_launch_ms / 1000.0) / 1e12, "peak": fp32_peak,
                            "unit": "TFLOP/s", "frac": flops / (per_launch_ms / 1000.0) / 1e12 / fp32_peak,
                            "flops_per_launch": flops,
                            "peak_source": "nominal FP32 (non-tensor): 148 SMs x 128 lanes x 2 x 1.965 GHz"}
        # compulsory bytes of a whole movie: every frame read once and its
        # spectrum written once, every spectrum read by the pair stage and by
        # the sum (twice more per realignment iteration), the image written
        S = plan.nsam * (plan.nsam // 2 + 1) * 8
        raw = host[0].numel() * host.element_size()
        b_movie = nz * (raw + 3 * S) + 2 * p.iter * nz * S + 4 * plan.nsam ** 2
        movie_gbs = b_movie / (ms_max / args.steps / 1000.0) / 1e9
        metric = METRIC if args.workload == "c2" else f"aligned frames/s at {nx}x{ny}x{nz}"
        line = {"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": (WORKLOAD if nz == 40 else f"profiling case: {nz} frames, else as c2")
                           if args.workload == "c2" else WORKLOADS_TEXT[args.workload],
                           "nsam": plan.nsam, "pairs": plan.npairs,
                           "l2": "inputs larger than L2 (570 MB frames, 2.2 GB spectra per movie), no flush",
                           "parallelism": f"replicas x{world}"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(host.numel()),
                        "d2h_bytes_per_step": int(image.numel() * 4),
                        "api": f"mc_batch_run, {args.lanes} lanes, frames and image in pinned host memory",
                        "latency_p50_ms": _pct(e2e_lat, 50), "latency_p99_ms": _pct(e2e_lat, 99),
                        "single_plan_value": nz * args.steps * world / (single_e2e_ms / 1000.0)},
                "api": f"mc_batch_run, {args.lanes} lanes, frames resident in HBM (bound in place)",
                "latency_p50_ms": _pct(dev_lat, 50), "latency_p99_ms": _pct(dev_lat, 99),
                "single_plan_value": nz * args.steps * world / (single_ms / 1000.0),
                "gpu_launches": launches, "roofline": roof,
                "movie_roofline": {"bytes_per_movie": b_movie, "achieved": movie_gbs, "peak": peak, "unit": "GB/s",
                                   "frac": movie_gbs / peak},
                "kernels": {k: {"ms_per_step": v["ms"] / prof_steps, "launches": v["launches"] // prof_steps,
                                "GBps": (v["bytes"] / (v["ms"] / 1000.0) / 1e9) if v["ms"] > 0 else None}
                            for k, v in stats.items()},
                "shift_rmse_vs_truth_px": truth_rmse,
                "clocks": clk.summary()}
        if world == 1 and not args.no_cpu_baseline and args.workload == "c2":
            v, parts = oracle_sample(seed=args.seed)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": "FP64 oracle, one frame forward + one pair + one frame sum at "
                                              "3710^2, scaled by P/F = 378/40; " +
                                              ", ".join(f"{k}={x:.2f}" for k, x in parts.items())}
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def _pct(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if xs else None


def run_c5(args):
    """Batch workload: 32 movies of mixed size and depth through the
    multi-lane batch runner (mc_batch_run) against the same runner with one
    lane (one movie at a time)."""
    import numpy as np
    import torch
    from motioncorr1exp_b200 import api, synth
    from motioncorr1exp_b200 import dist as D
    rank, world, local = D.world()
    if world > 1:
        raise SystemExit("the batch workload runs on one GPU per process; use --gpus 1")
    torch.cuda.set_device(local)
    jobs, means = synth.c5_jobs(seed=args.seed, n_movies=32, max_frames=80)
    base, base_host = [], []
    for g, (nx, ny) in enumerate(synth.C5_GEOMETRIES):
        fr, _ = synth.make_movie_torch(nx, ny, 80, mean=means[g], seed=args.seed + 10 + g, dtype="u8",
                                       kind="linear", speed=0.3, rw_sigma=0.5, device=f"cuda:{local}")
        base.append(fr)
        h = torch.empty(fr.shape, dtype=torch.uint8, pin_memory=True)
        h.copy_(fr)
        base_host.append(h)
    torch.cuda.synchronize()

    def movies(on_device):
        out = []
        for j in jobs:
            p = api.verify_params(api.Params(bin=1.0, FrameDistOffset=j["fod"], bfactor=150.0,
                                             CCPeakSearchDim=96, bAlignToMid=1, GPUNum=local), j["nframes"])
            g = j["geometry"]
            nx, ny = synth.C5_GEOMETRIES[g]
            fbytes = nx * ny
            n = (min(nx, ny) // 2) * 2
            m = {"params": p, "nx": nx, "ny": ny, "nz": j["nframes"], "mode": 0,
                 "image": np.empty((n, n), np.float32)}
            if on_device:
                m["device_ptr"] = base[g].data_ptr() + j["offset"] * fbytes
            else:
                m["frames"] = base_host[g].numpy()[j["offset"]: j["offset"] + j["nframes"]]
            out.append(m)
        return out

    nframes = sum(j["nframes"] for j in jobs)
    stream = torch.cuda.current_stream()

    def timed(batch, ms_list, on_device, reps):
        mv = movies(on_device)
        lat, comp = [], []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            res = batch.run(mv)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_list.append(e0.elapsed_time(e1))
            lat += [r["end_ms"] - r["start_ms"] for r in res]
            comp += [r["end_ms"] for r in res]
        return lat, comp

    out = {}
    for lanes in (1, args.lanes):
        with api.Batch(local, lanes) as b:
            for _ in range(args.warmup):
                b.run(movies(True))
            ms = []
            with ClockSampler(local) as clk:
                lat, comp = timed(b, ms, True, args.steps)
            e2e_ms = []
            b.run(movies(False))
            lat_h, comp_h = timed(b, e2e_ms, False, args.steps)
            out[lanes] = {"value": nframes * len(ms) / (sum(ms) / 1000.0),
                          "e2e": nframes * len(e2e_ms) / (sum(e2e_ms) / 1000.0),
                          "ms_per_batch": sum(ms) / len(ms),
                          "latency_p50_ms": _pct(lat, 50), "latency_p99_ms": _pct(lat, 99),
                          "completion_p50_ms": _pct(comp, 50), "completion_p99_ms": _pct(comp, 99),
                          "e2e_latency_p50_ms": _pct(lat_h, 50), "e2e_latency_p99_ms": _pct(lat_h, 99),
                          "device_gb": b.device_bytes / 1e9, "clocks": clk.summary()}
    best = out[args.lanes]
    line = {"metric": "aligned frames/s, batch of 32 movies (2048^2 / 3838x3710 / 4096^2, F~U[20,80])",
            "value": best["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": best["ms_per_batch"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "c5: 32 movies, geometry from {2048^2, 3838x3710, 4096^2}, F ~ U[20,80], "
                                   "fod in {2,4,7}, uint8, -bft 150 -pbx 96 -atm 1; frames are windows of one "
                                   "80-frame base movie per geometry (mean U[0.8,1.5])",
                       "frames_per_batch": nframes, "lanes": args.lanes,
                       "l2": "inputs larger than L2, no flush", "parallelism": "lanes on one GPU"},
            "e2e": {"value": best["e2e"], "unit": UNIT,
                    "h2d_bytes_per_step": int(sum(j["nframes"] * j["nx"] * j["ny"] for j in jobs)),
                    "d2h_bytes_per_step": int(sum(4 * ((min(j["nx"], j["ny"]) // 2) * 2) ** 2 for j in jobs))},
            "batch": {str(k): v for k, v in out.items()},
            "clocks": best["clocks"]}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--frames", type=int, default=0,
                    help="movie length (0: the workload's; fewer only for profiling captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the 40-frame 3838x3710 movie (headline); c1 1024^2x16 f32; c3 7676x7420x50 "
                         "uint8 -bin 2; c4 4096^2x60 f32 with 3 realignment iterations and the gradient "
                         "refinement; c5: the 32-movie batch")
    ap.add_argument("--lanes", type=int, default=2, help="batch lanes (each a host thread, stream and plans)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c5":
        run_c5(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
