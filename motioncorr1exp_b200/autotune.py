"""Autotuner of the pair-stage and forward-transform schedules (mc_schedule_set).

For a binned side n it times the pair stage (column stage + row stage) of a
synthetic movie under every split n = P*Q the register-codelet kernel takes
and several pair-per-CTA counts, and keeps the fastest; then, with that pair
schedule, the forward transforms of the movie under every forked-stream
count (1, 2, 4, 8) and radix-53 pairing of the row and column passes (one or
two output pairs per loop pass), and keeps the fastest.  Results are cached
as JSON keyed by GPU name and n:

    {"NVIDIA B200": {"3710": {"pair_q": 35, "pairs_per_cta": 32, "pair_variant": 0,
                              "ms": ..., "trials": [...]}}}

    python -m motioncorr1exp_b200.autotune --n 2048 3710 4096 [--out FILE]

`load()` installs the cached entries of the current GPU into the library;
api.Plan calls it once before the first plan is created (set MC_SCHEDULES=0
to keep the built-in choices).
"""
from __future__ import annotations

import argparse
import json
import os
from typing import Optional

from . import api

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PATH = os.path.join(HERE, "tune", "schedules.json")
PAIRS_PER_CTA = (8, 16, 32, 64)


def gpu_name(device: int = 0) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def _time_pairs(n: int, frames, params: api.Params, reps: int) -> tuple[float, int]:
    nz = frames.shape[0]
    with api.Plan(params, n, n, nz, 0) as pl:
        pl.load_frames_device(frames.data_ptr(), 0, nz)
        pl.forward()
        pl.pairs()                      # warm-up (function attributes, caches)
        pl.reset_stats()
        pl.set_profiling(True)
        for _ in range(reps):
            pl.pairs()
        pl.set_profiling(False)
        st = pl.kernel_stats()
        ms = (st["k_pair_cols"]["ms"] + st["k_pair_rows"]["ms"]) / reps
        return ms, pl.info["prune_q"]


def _time_forward(n: int, frames, params: api.Params, reps: int) -> float:
    nz = frames.shape[0]
    with api.Plan(params, n, n, nz, 0) as pl:
        pl.load_frames_device(frames.data_ptr(), 0, nz)
        pl.forward()                    # warm-up
        ts = []
        for _ in range(reps):
            pl.forward()
            ts.append(pl.timings()["forward_ms"])
        return float(sorted(ts)[len(ts) // 2])


FWD_STREAMS = (1, 2, 4, 8)


def tune(n: int, box: int = 96, nframes: int = 16, fod: int = 2, reps: int = 3, device: int = 0,
         seed: int = 0) -> dict:
    """Times every candidate schedule for side n; returns the best entry with
    the list of trials.  Leaves the library's schedule table as it found it
    apart from the entry for n, which is set to the winner."""
    import torch
    from . import synth
    frames, _ = synth.make_movie_torch(n, n, nframes, mean=1.2, seed=seed, dtype="u8", kind="linear",
                                       speed=0.3, rw_sigma=0.5, device=f"cuda:{device}")
    torch.cuda.synchronize()
    params = api.verify_params(api.Params(CCPeakSearchDim=box, FrameDistOffset=fod, GPUNum=device), nframes)
    trials = []
    for q in api.schedule_candidates(n):
        for ppc in PAIRS_PER_CTA:
            api.schedule_set(n, pair_q=q, pairs_per_cta=ppc)
            ms, used_q = _time_pairs(n, frames, params, reps)
            if used_q == q:
                trials.append({"pair_q": q, "pairs_per_cta": ppc, "pair_variant": 0, "ms": ms})
    if not trials:
        raise RuntimeError(f"no register-codelet split for n={n}")
    best = min(trials, key=lambda t: t["ms"])
    # forward transforms under the chosen pair schedule (pairing only matters
    # where the length has a radix-53 step; the others time the same)
    fwd = []
    for fs in FWD_STREAMS:
        for rp in (1, 2):
            for cp in (1, 2):
                api.schedule_set(n, pair_q=best["pair_q"], pairs_per_cta=best["pairs_per_cta"], fwd_streams=fs,
                                 fwd_rows_pairing=rp, fwd_cols_pairing=cp)
                fwd.append({"fwd_streams": fs, "fwd_rows_pairing": rp, "fwd_cols_pairing": cp,
                            "ms": _time_forward(n, frames, params, reps)})
    bf = min(fwd, key=lambda t: t["ms"])
    # keep the built-in forward schedule (4 streams, rows and columns paired)
    # unless another is more than 1 % faster: the trials time one plan alone,
    # and a difference inside the noise is no reason to change what the
    # batch lanes interleave with
    base = next(t for t in fwd if (t["fwd_streams"], t["fwd_rows_pairing"], t["fwd_cols_pairing"]) == (4, 2, 2))
    if base["ms"] <= 1.01 * bf["ms"]:
        bf = base
    api.schedule_set(n, pair_q=best["pair_q"], pairs_per_cta=best["pairs_per_cta"],
                     pair_variant=best["pair_variant"], fwd_streams=bf["fwd_streams"],
                     fwd_rows_pairing=bf["fwd_rows_pairing"], fwd_cols_pairing=bf["fwd_cols_pairing"])
    return {**best, "fwd_streams": bf["fwd_streams"], "fwd_rows_pairing": bf["fwd_rows_pairing"],
            "fwd_cols_pairing": bf["fwd_cols_pairing"], "fwd_ms": bf["ms"],
            "box": box, "pairs": sum(max(0, nframes - (i + max(1, nframes // 2 - fod))) for i in range(nframes)),
            "trials": trials, "fwd_trials": fwd}


def save(results: dict, gpu: str, path: str = DEFAULT_PATH) -> None:
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data.setdefault(gpu, {}).update({str(n): r for n, r in results.items()})
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
        f.write("\n")


def load(path: Optional[str] = None, gpu: Optional[str] = None) -> int:
    """Installs the cached schedules of this GPU; returns how many."""
    path = path or DEFAULT_PATH
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        data = json.load(f)
    if gpu is None:
        try:
            gpu = gpu_name()
        except Exception:
            return 0
    count = 0
    for n, r in data.get(gpu, {}).items():
        try:
            api.schedule_set(int(n), pair_q=int(r["pair_q"]), pairs_per_cta=int(r["pairs_per_cta"]),
                             pair_variant=int(r.get("pair_variant", 0)), fwd_streams=int(r.get("fwd_streams", 0)),
                             fwd_rows_pairing=int(r.get("fwd_rows_pairing", 0)),
                             fwd_cols_pairing=int(r.get("fwd_cols_pairing", 0)))
            count += 1
        except Exception:
            continue   # an entry the compiled kernels of libmc no longer take
    return count


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, nargs="+", default=[2048, 3710, 4096])
    ap.add_argument("--box", type=int, default=96)
    # 40 frames with fod 7: the 378 pairs of the 40-frame benchmark movie, so
    # the pair batch (and the L2 reuse across pairs) has the benchmark's shape
    ap.add_argument("--frames", type=int, default=40)
    ap.add_argument("--fod", type=int, default=7)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_PATH)
    a = ap.parse_args()
    api.schedule_clear()
    res = {}
    for n in a.n:
        res[n] = tune(n, a.box, a.frames, fod=a.fod, reps=a.reps, device=a.device)
        t = res[n]
        print(json.dumps({"n": n, "pair_q": t["pair_q"], "pairs_per_cta": t["pairs_per_cta"], "ms": t["ms"],
                          "trials": [(x["pair_q"], x["pairs_per_cta"], round(x["ms"], 4)) for x in t["trials"]],
                          "fwd": [t["fwd_streams"], t["fwd_rows_pairing"], t["fwd_cols_pairing"], t["fwd_ms"]],
                          "fwd_trials": [(x["fwd_streams"], x["fwd_rows_pairing"], x["fwd_cols_pairing"],
                                          round(x["ms"], 4)) for x in t["fwd_trials"]]}),
              flush=True)
    save(res, gpu_name(a.device), a.out)


if __name__ == "__main__":
    main()
