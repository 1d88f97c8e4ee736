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
MOVIE_FRAMES, MOVIE_PAIRS = 40, 378
STEP_FRAMES = 2                                      # one step = 1/20 of the movie
STEP_PAIRS = MOVIE_PAIRS * STEP_FRAMES / MOVIE_FRAMES  # 18.9 pairs


def oracle_step(F, mask, nu, frames_raw, k):
    """One step of the FP64 oracle's c2 workload, timed: 1/20 of the movie =
    the forward transforms of 2 frames, 19 pair correlations + sub-pixel
    peaks (their time scaled by 18.9/19: 378 pairs / 40 frames x 2) and 2
    frames of the phase-shift sum.  Returns (seconds, timed parts)."""
    from oracle import mc_oracle as O
    t0 = time.perf_counter()
    Fk = [O.forward_spectrum(O.decode_frame(frames_raw[(k + i) % len(frames_raw)], 0), 0, 0, nu, nu)
          for i in range(STEP_FRAMES)]
    t1 = time.perf_counter()
    npair = int(math.ceil(STEP_PAIRS))
    for i in range(npair):
        O.find_shift(O.cc_box(O.cc_map(F[i % len(F)], F[(i + 13) % len(F)], mask, nu), nu, 96), nu, 0)
    t2 = time.perf_counter()
    S = O.phase_shift(Fk[0], 0.3, -0.2)
    S = S + O.phase_shift(Fk[1], -0.1, 0.4)
    t3 = time.perf_counter()
    pair_s = (t2 - t1) * STEP_PAIRS / npair
    return (t1 - t0) + pair_s + (t3 - t2), {"fwd_s": t1 - t0, "pairs_s": pair_s, "sum_s": t3 - t2}


def c2_host_movie(seed, nframes):
    """The c2 movie on the host: generated by the same seeded model as the GPU
    arm (on the GPU when one is visible, else with numpy)."""
    from motioncorr1exp_b200 import synth
    try:
        import torch
        if torch.cuda.is_available():
            fr, truth = synth.make_movie_torch(3838, 3710, nframes, mean=1.2, seed=seed, dtype="u8", kind="linear",
                                               speed=0.3, rw_sigma=0.5, device="cuda")
            out = fr.cpu().numpy()
            del fr
            torch.cuda.empty_cache()
            return out, truth
    except Exception:
        pass
    mv = synth.make_movie(3838, 3710, nframes, mean=1.2, seed=seed, dtype="u8", speed=0.3, rw_sigma=0.5)
    return mv.frames, mv.truth


def run_reference(args):
    """The reference algorithm's CPU implementation (the FP64 oracle port) on
    the host cores: K timed steps of 1/20 of the c2 movie each, then one
    whole-movie run as a check of the per-step model."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import mc_oracle as O
    cores = os.cpu_count() or 1
    frames, _ = c2_host_movie(args.seed, MOVIE_FRAMES)
    nu = O.verify_crop_size(3838, 3710, 0, 0, 0, 1.0)
    mask = O.bfactor_mask(nu, 150.0)
    F = [O.forward_spectrum(O.decode_frame(frames[k], 0), 0, 0, nu, nu) for k in range(2)]
    times, parts = [], []
    for i in range(args.warmup + args.steps):
        t, pr = oracle_step(F, mask, nu, frames, 2 * i)
        if i >= args.warmup:
            times.append(t)
            parts.append(pr)
    step_s = statistics.median(times)
    value = STEP_FRAMES / step_s
    check = {}
    if not args.no_oracle_check:
        p = O.verify_para(O.Params(FrameDistOffset=7, bfactor=150.0, CCPeakSearchDim=96, bAlignToMid=1), 40)
        t0 = time.perf_counter()
        O.align_movie(frames, 0, p)
        whole = time.perf_counter() - t0
        check = {"whole_movie_s": whole, "whole_movie_frames_per_s": MOVIE_FRAMES / whole,
                 "step_model_frames_per_s": value}
    sample = (f"FP64 oracle port (numpy/scipy pocketfft on {cores} host threads); one step = 1/20 of the c2 movie: "
              f"the forward transforms of 2 frames, 19 pair correlations + FindShift (time scaled by 18.9/19) and "
              f"2 frames of the phase-shift sum; value = 2 frames / median step time")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * step_s,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                             "parts_s": {k: statistics.median(x[k] for x in parts) for k in parts[0]}},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if check:
        line["whole_movie_check"] = check
    print(json.dumps(line), flush=True)


def oracle_check(host_frames, mode, p, g, nps):
    """FP64 oracle of the whole movie (outside every timed region) and the
    parity metrics of the GPU run ``g`` against it."""
    from oracle import mc_oracle as O
    from oracle import parity
    op = O.Params(**{k: getattr(p, k) for k in O.Params.__dataclass_fields__})
    t0 = time.perf_counter()
    ref = O.align_movie(host_frames, mode, op, keep_boxes=True)
    m = parity.compare_alignment(g, ref, nps)
    return {"shift_rmse_vs_oracle_px": m["shift_rmse_vs_oracle_px"],
            "shift_max_diff_vs_oracle_px": m["shift_max_diff_px"],
            "sum_rel_l2_vs_oracle": m.get("sum_rel_l2_vs_oracle"),
            "pair_list_equal": m["pair_list_equal"], "kept_pairs_equal": m.get("kept_equal"),
            "peak_flips": m["peak_flips"], "grid_flips": m["grid_flips"],
            "flips_unexplained_by_near_ties": len(m["violations"]),
            "oracle_s": time.perf_counter() - t0}


def oracle_check_refined(host_frames, mode, p_plain, g_plain, g_refined, nps):
    """c4: the FP64 oracle of the whole movie with -itr 3 (outside every timed
    region).  The plain path (-ref 0) is compared like the other workloads;
    the refined shifts have no counterpart in the reference's pipeline, so
    they are checked as a fixed point of the FP64 block-Newton refinement
    (the largest step the oracle takes from them) and the refined sum against
    the oracle's sum at the same shifts."""
    import numpy as np
    from oracle import mc_oracle as O
    from oracle import parity
    op = O.Params(**{k: getattr(p_plain, k) for k in O.Params.__dataclass_fields__})
    t0 = time.perf_counter()
    ref = O.align_movie(host_frames, mode, op, keep_boxes=True, keep_spectra=True)
    m = parity.compare_alignment(g_plain, ref, nps)
    steps = O.newton_steps(ref.spectra, -g_refined["frame_shifts"], float(p_plain.bfactor))
    fs = g_refined["frame_shifts"][:, 0] + 1j * g_refined["frame_shifts"][:, 1]
    _, img = O.corrected_sum(ref.spectra, np.diff(fs), op, 0, len(fs))
    return {"plain": {"shift_rmse_vs_oracle_px": m["shift_rmse_vs_oracle_px"],
                      "shift_max_diff_vs_oracle_px": m["shift_max_diff_px"],
                      "sum_rel_l2_vs_oracle": m.get("sum_rel_l2_vs_oracle"),
                      "pair_list_equal": m["pair_list_equal"], "kept_pairs_equal": m.get("kept_equal"),
                      "peak_flips": m["peak_flips"], "grid_flips": m["grid_flips"],
                      "flips_unexplained_by_near_ties": len(m["violations"])},
            "refined": {"largest_fp64_newton_step_px": float(np.max(np.hypot(steps[:, 0], steps[:, 1]))),
                        "sum_rel_l2_vs_oracle_at_refined_shifts": parity.rel_l2(g_refined["image"], img)},
            "oracle_s": time.perf_counter() - t0}


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
    if args.storage == "f16":
        # integer counts held as IEEE half (MRC2014 mode 12): exact below 2048
        if mode != 2:
            raise SystemExit("--storage f16 applies to float32 workloads (c1, c4)")
        if bool((frames != frames.round()).any()) or float(frames.abs().max()) > 2048:
            raise SystemExit("--storage f16 needs integer counts below 2048")
        frames = frames.half()
        mode = api.MODE_F16
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

    # ---- the same K movies as one CUDA graph per batch (mc_batch_set_graph:
    # lanes as graph branches, one launch, one synchronisation); the graph is
    # captured in the warm-up and relaunched in the timed call
    graph_ms = None
    if p.iter == 0 and not p.refine:
        gb = api.Batch(local, args.lanes, graph=True)
        for _ in range(max(1, args.warmup // 2)):
            gb.run(dev)
        graph_ms, _ = timed(lambda: gb.run(dev))
        gb.close()

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

    # host->device copy bandwidth from pinned memory (the bound of the e2e
    # figure: every step uploads its frames): 1 GiB copied 5 times, best
    h2d_src = torch.empty(1 << 30, dtype=torch.uint8, pin_memory=True)
    h2d_dst = torch.empty(1 << 30, dtype=torch.uint8, device=f"cuda:{local}")
    h2d_s = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        h2d_dst.copy_(h2d_src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        h2d_s.append(e0.elapsed_time(e1) / 1000.0)
    h2d_gbs = (1 << 30) / min(h2d_s) / 1e9
    del h2d_src, h2d_dst
    # the single-plan form of the same call, one movie at a time
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    single_e2e_ms, _ = timed(lambda: [step_e2e() for _ in range(args.steps)])

    # shifts come in binned pixels (nsam / nsam_unbin of a raw pixel)
    to_binned = plan.nsam / plan.info["nsam_unbin"]

    def rmse_truth(sh):
        return float(np.sqrt(np.mean(np.sum((sh + to_binned * (truth - truth[0])) ** 2, axis=1))))
    truth_rmse = rmse_truth(shifts)

    # ---- one movie's full result (outside every timed region) for the
    # checks against the FP64 oracle below
    g_img = plan.run(want_image=True)
    g_res = {"image": g_img, "frame_shifts": plan.frame_shifts(), **plan.pair_results(), **plan.ki()}

    # ---- c4: the gradient refinement against the plain peak fit on the same
    # movie (north-star target: lower ground-truth RMSE at <= 1.3x the time)
    refine_cmp = None
    g_plain, p_plain = None, None
    if args.workload == "c4":
        p_plain = api.Params(**{**vars(p), "refine": 0})
        with api.Plan(p_plain, nx, ny, nz, mode) as pp:
            pp.load_frames_device(frames.data_ptr(), 0, nz)
            for _ in range(max(1, args.warmup // 2)):
                pp.run(want_image=False)
            plain_ms, _ = timed(lambda: [pp.run(want_image=False) for _ in range(args.steps)])
            plain_shifts = pp.frame_shifts()
            g_plain = {"image": pp.run(want_image=True), "frame_shifts": pp.frame_shifts(), **pp.pair_results(),
                       **pp.ki()}
        refine_cmp = {"plain_ms_per_movie": plain_ms / args.steps, "refined_ms_per_movie": single_ms / args.steps,
                      "time_ratio": single_ms / plain_ms, "truth_rmse_plain_px": rmse_truth(plain_shifts),
                      "truth_rmse_refined_px": truth_rmse,
                      "target": "refined RMSE lower than plain at <= 1.3x its time"}

    if rank == 0:
        value = nz * args.steps * world / (ms_max / 1000.0)
        e2e_value = nz * args.steps * world / (e2e_ms / 1000.0)
        # frames/s if every movie's upload ran back to back at the pinned copy bandwidth
        h2d_bound = world * nz / (host.numel() * host.element_size() / (h2d_gbs * 1e9))
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
                           "frame_storage": ("IEEE half (MRC mode 12), exact for these counts"
                                             if args.storage == "f16" else "file pixel type"),
                           "l2": (f"inputs larger than L2 ({nz * raw / 1e6:.0f} MB frames, "
                                  f"{nz * S / 1e9:.1f} GB spectra per movie), no flush"),
                           "parallelism": f"replicas x{world}"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(host.numel() * host.element_size()),
                        "h2d_roofline": {"pinned_h2d_gbs": h2d_gbs,
                                         "bound_frames_per_s": h2d_bound,
                                         "frac": e2e_value / h2d_bound,
                                         "note": "upload of each movie's frames at the measured pinned copy bandwidth"},
                        "d2h_bytes_per_step": int(image.numel() * 4),
                        "api": f"mc_batch_run, {args.lanes} lanes, frames and image in pinned host memory",
                        "latency_p50_ms": _pct(e2e_lat, 50), "latency_p99_ms": _pct(e2e_lat, 99),
                        "single_plan_value": nz * args.steps * world / (single_e2e_ms / 1000.0)},
                "api": f"mc_batch_run, {args.lanes} lanes, frames resident in HBM (bound in place)",
                "latency_p50_ms": _pct(dev_lat, 50), "latency_p99_ms": _pct(dev_lat, 99),
                "single_plan_value": nz * args.steps * world / (single_ms / 1000.0),
                "single_graph_value": (nz * args.steps * world / (graph_ms / 1000.0)) if graph_ms else None,
                "gpu_launches": launches, "roofline": roof,
                "movie_roofline": {"bytes_per_movie": b_movie, "achieved": movie_gbs, "peak": peak, "unit": "GB/s",
                                   "frac": movie_gbs / peak},
                "kernels": {k: {"ms_per_step": v["ms"] / prof_steps, "launches": v["launches"] // prof_steps,
                                "GBps": (v["bytes"] / (v["ms"] / 1000.0) / 1e9) if v["ms"] > 0 else None}
                            for k, v in stats.items()},
                "shift_rmse_vs_truth_px": truth_rmse,
                "clocks": clk.summary()}
        if refine_cmp:
            line["refinement_vs_plain"] = refine_cmp
        host_np_all = host.numpy()
        if world == 1 and not args.no_cpu_baseline and args.workload == "c2":
            from oracle import mc_oracle as O
            nu = plan.info["nsam_unbin"]
            mask = O.bfactor_mask(nu, 150.0)
            F = [O.forward_spectrum(O.decode_frame(host_np_all[k], 0), 0, 0, nu, nu) for k in range(2)]
            ts = [oracle_step(F, mask, nu, host_np_all, 2 * i)[0] for i in range(6)][1:]
            v = STEP_FRAMES / statistics.median(ts)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": f"FP64 oracle port on {os.cpu_count() or 1} host threads, 5 steps of "
                                              "1/20 of this movie each (2 frame forwards, 18.9 pair "
                                              "correlations + FindShift, 2 frames of the sum; one warm-up "
                                              f"step); median step {statistics.median(ts):.2f} s"}
        if world == 1 and args.workload == "c2" and not args.no_batch_c5:
            # the batch workload beside the headline: 32 mixed movies, one lane
            # (one movie at a time) against --lanes lanes.  Three warm-up
            # batches, as in --workload c5: the lanes take movies in arrival
            # order, so a lane's plans capture the CUDA graph of a frame
            # configuration (32 of them here) the first time they run it.
            r5 = c5_measure(local, args.seed, (1, args.lanes), 2, 3)
            line["batch_c5"] = {"workload": C5_WORKLOAD, "frames_per_batch": r5["frames_per_batch"],
                                "lanes": {str(k): dict(v) for k, v in r5["lanes"].items()}}
        if world == 1 and not args.no_oracle_check and args.workload in ("c1", "c2", "c3"):
            line["vs_oracle"] = oracle_check(host_np_all, mode, p, g_res, p.NoisePeakSize)
            line["shift_rmse_vs_oracle_px"] = line["vs_oracle"]["shift_rmse_vs_oracle_px"]
            line["sum_rel_l2_vs_oracle"] = line["vs_oracle"]["sum_rel_l2_vs_oracle"]
            line["pair_flips_vs_oracle"] = line["vs_oracle"]["peak_flips"] + line["vs_oracle"]["grid_flips"]
        if world == 1 and not args.no_oracle_check and args.workload == "c4" and g_plain is not None:
            vo = oracle_check_refined(host_np_all, mode, p_plain, g_plain, g_res, p.NoisePeakSize)
            line["vs_oracle"] = vo
            line["shift_rmse_vs_oracle_px"] = vo["plain"]["shift_rmse_vs_oracle_px"]
            line["sum_rel_l2_vs_oracle"] = vo["refined"]["sum_rel_l2_vs_oracle_at_refined_shifts"]
            line["pair_flips_vs_oracle"] = vo["plain"]["peak_flips"] + vo["plain"]["grid_flips"]
            line["refined_newton_step_vs_oracle_px"] = vo["refined"]["largest_fp64_newton_step_px"]
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def _pct(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if xs else None


def c5_measure(local, seed, lanes_list, steps, warmup):
    """The batch workload (32 movies of mixed size and depth, frames windows
    of one 80-frame base movie per geometry) through the batch runner with
    each lane count of ``lanes_list``: frames/s with the frames in HBM and
    from pinned host memory, per-movie latency and completion percentiles."""
    import numpy as np
    import torch
    from motioncorr1exp_b200 import api, synth
    jobs, means = synth.c5_jobs(seed=seed, n_movies=32, max_frames=80)
    base, base_host = [], []
    for g, (nx, ny) in enumerate(synth.C5_GEOMETRIES):
        fr, _ = synth.make_movie_torch(nx, ny, 80, mean=means[g], seed=seed + 10 + g, dtype="u8",
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
    for lanes in lanes_list:
        with api.Batch(local, lanes) as b:
            for _ in range(warmup):
                b.run(movies(True))
            ms = []
            with ClockSampler(local) as clk:
                lat, comp = timed(b, ms, True, steps)
            e2e_ms = []
            b.run(movies(False))
            lat_h, comp_h = timed(b, e2e_ms, False, steps)
            out[lanes] = {"value": nframes * len(ms) / (sum(ms) / 1000.0),
                          "e2e": nframes * len(e2e_ms) / (sum(e2e_ms) / 1000.0),
                          "ms_per_batch": sum(ms) / len(ms),
                          "latency_p50_ms": _pct(lat, 50), "latency_p99_ms": _pct(lat, 99),
                          "completion_p50_ms": _pct(comp, 50), "completion_p99_ms": _pct(comp, 99),
                          "e2e_latency_p50_ms": _pct(lat_h, 50), "e2e_latency_p99_ms": _pct(lat_h, 99),
                          "device_gb": b.device_bytes / 1e9, "clocks": clk.summary()}
    del base, base_host
    torch.cuda.empty_cache()
    return {"frames_per_batch": nframes, "jobs": jobs, "lanes": out}


C5_WORKLOAD = ("c5: 32 movies, geometry from {2048^2, 3838x3710, 4096^2}, F ~ U[20,80], fod in {2,4,7}, uint8, "
               "-bft 150 -pbx 96 -atm 1; frames are windows of one 80-frame base movie per geometry "
               "(mean U[0.8,1.5])")


def run_c5(args):
    """Batch workload: 32 movies of mixed size and depth through the
    multi-lane batch runner (mc_batch_run) against the same runner with one
    lane (one movie at a time)."""
    import torch
    from motioncorr1exp_b200 import dist as D
    rank, world, local = D.world()
    if world > 1:
        raise SystemExit("the batch workload runs on one GPU per process; use --gpus 1")
    torch.cuda.set_device(local)
    r = c5_measure(local, args.seed, (1, args.lanes), args.steps, args.warmup)
    jobs, nframes, out = r["jobs"], r["frames_per_batch"], r["lanes"]
    best = out[args.lanes]
    line = {"metric": "aligned frames/s, batch of 32 movies (2048^2 / 3838x3710 / 4096^2, F~U[20,80])",
            "value": best["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": best["ms_per_batch"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": C5_WORKLOAD, "frames_per_batch": nframes, "lanes": args.lanes,
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
    ap.add_argument("--no-batch-c5", action="store_true",
                    help="skip the 32-movie batch workload reported beside the c2 line")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the whole-movie FP64 oracle run that checks the result (and the step model)")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the 40-frame 3838x3710 movie (headline); c1 1024^2x16 f32; c3 7676x7420x50 "
                         "uint8 -bin 2; c4 4096^2x60 f32 with 3 realignment iterations and the gradient "
                         "refinement; c5: the 32-movie batch")
    ap.add_argument("--lanes", type=int, default=2, help="batch lanes (each a host thread, stream and plans)")
    ap.add_argument("--storage", default="native", choices=["native", "f16"],
                    help="f16: float32 count frames held as IEEE half (MRC mode 12) on the device and the host")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c5":
        run_c5(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
