"""Full-size parity: the benchmark movies through the CUDA path (C ABI) against
the FP64 oracle, every frame and every pair.

  c2  40 x 3838x3710 uint8, -fod 7 -atm 1 (crop 3710: radix 53), 378 pairs
  c3  50 x 7676x7420 uint8, -bin 2 (7420 -> 3710 Fourier crop), 378 pairs
  c4  60 x 4096^2 float32, -itr 3 -ith 0.01, 528 pairs; plain (-ref 0) and
      with the gradient refinement (-ref 1)

Bars (oracle/parity.py): identical pair list; integer peaks and 1/32-px pair
shifts identical except near-ties that the oracle's own CC values explain;
frame shifts within 0.01 px; sum within 1e-5 relative L2.  With -ref 1 the
refined shifts have no counterpart in the oracle's pipeline; they must sit
within 0.01 px of a fixed point of the FP64 refinement (the oracle's
block-Newton step from them, O.newton_steps, is at most 0.01 px per frame).
Synthetic movies come from the seeded generator the benchmark uses
(motioncorr1exp_b200.synth.make_movie_torch).
"""
import numpy as np
import pytest

from motioncorr1exp_b200 import api, synth
from oracle import mc_oracle as O
from oracle import parity

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def to_oparams(p: api.Params) -> O.Params:
    return O.Params(**{k: getattr(p, k) for k in O.Params.__dataclass_fields__})


def make(name, seed=0):
    import torch
    w = dict(synth.WORKLOADS[name])
    flags = dict(w.pop("flags"))
    frames, truth = synth.make_movie_torch(w["nx"], w["ny"], w["nframes"], mean=w["mean"], seed=seed,
                                           dtype=w["dtype"], kind=w["kind"], speed=w.get("speed", 0.4),
                                           rw_sigma=w.get("rw_sigma", 0.3), amp=w.get("amp", 1.5),
                                           period=w.get("period", 20.0), device="cuda")
    torch.cuda.synchronize()
    return frames, frames.cpu().numpy(), truth, flags, w


def run_gpu(frames_dev, p, nx, ny, nz, mode):
    with api.Plan(p, nx, ny, nz, mode) as pl:
        pl.load_frames_device(frames_dev.data_ptr(), 0, nz)
        img = pl.run()
        return {"image": img, "frame_shifts": pl.frame_shifts(), **pl.pair_results(), **pl.ki(),
                "nsam": pl.nsam, "nsam_unbin": pl.info["nsam_unbin"]}


def truth_rmse(shifts, truth, scale):
    d = shifts + scale * (truth - truth[0])
    return float(np.sqrt(np.mean(np.sum(d * d, axis=1))))


def check(name, g, ref, p):
    m = parity.compare_alignment(g, ref, p.NoisePeakSize)
    print(f"{name}: {m['pairs']} pairs, peak flips {m['peak_flips']}, grid flips {m['grid_flips']}, "
          f"max frame-shift diff {m['shift_max_diff_px']:.2e} px, RMSE vs oracle "
          f"{m['shift_rmse_vs_oracle_px']:.2e} px, sum rel L2 {m.get('sum_rel_l2_vs_oracle', float('nan')):.2e}")
    assert not m["violations"], m["violations"][:10]
    assert m["peak_flips"] + m["grid_flips"] <= max(1, m["pairs"] // 50)
    return m


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_fullsize_plain(gpu, name):
    frames, host, truth, flags, w = make(name)
    nz = w["nframes"]
    mode = 0 if w["dtype"] == "u8" else 2
    p = api.verify_params(api.Params(**flags), nz)
    g = run_gpu(frames, p, w["nx"], w["ny"], nz, mode)
    del frames
    ref = O.align_movie(host, mode, to_oparams(p), keep_boxes=True)
    check(name, g, ref, p)
    assert g["kept"].tolist() == [int(x) for x in ref.goodlist]


@pytest.fixture(scope="module")
def c4():
    frames, host, truth, flags, w = make("c4")
    nz = w["nframes"]
    p0 = api.verify_params(api.Params(**flags), nz)
    g0 = run_gpu(frames, p0, w["nx"], w["ny"], nz, 2)
    p1 = api.verify_params(api.Params(**flags, refine=1), nz)
    g1 = run_gpu(frames, p1, w["nx"], w["ny"], nz, 2)
    del frames
    ref = O.align_movie(host, 2, to_oparams(p0), keep_boxes=True, keep_spectra=True)
    return {"p": p0, "g0": g0, "g1": g1, "ref": ref, "truth": truth}


def test_fullsize_c4_iterations(gpu, c4):
    check("c4 -itr 3", c4["g0"], c4["ref"], c4["p"])


def test_fullsize_c4_refined(gpu, c4):
    g1, ref = c4["g1"], c4["ref"]
    steps = O.newton_steps(ref.spectra, -g1["frame_shifts"], float(c4["p"].bfactor))
    worst = float(np.max(np.hypot(steps[:, 0], steps[:, 1])))
    plain = truth_rmse(c4["g0"]["frame_shifts"], c4["truth"], 1.0)
    refined = truth_rmse(g1["frame_shifts"], c4["truth"], 1.0)
    print(f"c4 -ref 1: largest FP64 Newton step from the refined shifts {worst:.2e} px; "
          f"truth RMSE plain {plain:.4f} px, refined {refined:.4f} px")
    assert worst <= parity.SHIFT_TOL
    # the sum at the refined shifts against the oracle's sum at the same shifts
    fs = g1["frame_shifts"][:, 0] + 1j * g1["frame_shifts"][:, 1]
    _, img = O.corrected_sum(ref.spectra, np.diff(fs), to_oparams(c4["p"]), 0, len(fs))
    assert parity.rel_l2(g1["image"], img) <= parity.IMAGE_RTOL
