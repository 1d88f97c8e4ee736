"""Spectrum slots (mc_plan_create_slots): a plan that holds fewer spectra
than frames recomputes a frame's forward transform whenever a stage needs a
spectrum it gave up -- the pair stage in blocks of slots/2 frames, the sums,
the frame-to-sum iterations (DFAlign.cu:950-1071) and the refinement
objective with its adjoint pass in chunks of `slots` frames.  The reference
holds every spectrum in host memory instead (hbuf / hbuf2, DFAlign.cu:545-546).

Every result must equal the resident plan's bit for bit: the same kernels
run on the same spectra and the sums accumulate in the same frame order.
Covered: odd and even slot counts, -itr with -ref 1, Fourier-crop binning
(the forward pass's shared row buffer), the two spectrum sets of two-frame
references, a size outside the two-level transforms (the fused sum kernel),
the extra sum outputs, the objective, the automatic choice under a device
budget (mc_debug_device_budget) and the batch runner.
"""
import numpy as np
import pytest

from motioncorr1exp_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu

KEEP_FREE = 256 << 20  # what the automatic choice leaves free


def _run(mv, mode, p, slots, refs=None, extra=False):
    nz, ny, nx = mv.frames.shape
    with api.Plan(p, nx, ny, nz, mode, spectrum_slots=slots) as pl:
        if refs:
            pl.set_refs(**refs)
        pl.load_frames(mv.frames[pl.info["nstart"]: pl.info["nend"] + 1])
        out = {"image": pl.run(), "shifts": pl.frame_shifts(), **pl.pair_results(), "boxes": pl.boxes(),
               "means": pl.frame_means(), "slots": pl.spectrum_slots}
        if extra:
            sh, first, last = pl.sum_shifts()
            out["raw"] = pl.raw_sum()
            out["part"] = pl.sum_to(first + (last - first) // 2 + pl.info["nstart"])
            out["frame"] = pl.corrected_frame(last + pl.info["nstart"])
            for kind in ("raw_fft", "corr_sum", "corr_fft"):
                out["ql_" + kind] = pl.quicklook(kind)
            out["spec3"] = pl.spectrum(3)
            if pl.info["two_sets"]:
                out["spec3b"] = pl.spectrum(3, 1)
        out["recomputes"] = pl.forward_recomputes
    return out


def _assert_same(a, b):
    for k in a:
        if k in ("slots", "recomputes"):
            continue
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)


CASES = {
    # name: (nx, ny, nz, mode/dtype, params, slots)
    "u8_itr2_ref1_slots4": (530, 520, 14, "u8", dict(crop_nsam=512, FrameDistOffset=2, iter=2, refine=1), 4),
    "u8_itr2_ref1_slots5": (530, 520, 14, "u8", dict(crop_nsam=512, FrameDistOffset=2, iter=2, refine=1), 5),
    "f32_bin2_slots4": (1060, 1040, 9, "f32", dict(crop_nsam=1024, bin=2.0, iter=1), 4),
    "u8_n500_fused_sum_slots6": (520, 510, 10, "u8", dict(crop_nsam=500, iter=1), 6),
}


@pytest.mark.parametrize("name", list(CASES))
def test_slots_equal_resident(gpu, name):
    nx, ny, nz, dt, kw, slots = CASES[name]
    mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=171 + nz, dtype=dt, speed=0.6, rw_sigma=0.4)
    mode = 0 if dt == "u8" else 2
    p = api.verify_params(api.Params(CCPeakSearchDim=64, **kw), nz)
    full = _run(mv, mode, p, None, extra=True)
    held = _run(mv, mode, p, slots, extra=True)
    assert full["slots"] == 0 and full["recomputes"] == 0
    assert held["slots"] == slots
    assert held["recomputes"] > 0
    _assert_same(full, held)


def test_slots_two_spectrum_sets(gpu):
    nx, ny, nz = 530, 520, 10
    mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=181, dtype="u8", speed=0.6, rw_sigma=0.4)
    rng = np.random.default_rng(5)
    refs = {"dark": rng.normal(0.2, 0.02, (ny, nx)).astype(np.float32),
            "dark2": rng.normal(0.2, 0.02, (ny, nx)).astype(np.float32),
            "norm": rng.normal(1.0, 0.05, (ny, nx)).astype(np.float32),
            "norm2": rng.normal(1.0, 0.05, (ny, nx)).astype(np.float32)}
    p = api.verify_params(api.Params(crop_nsam=512, CCPeakSearchDim=64, iter=1), nz)
    full = _run(mv, 0, p, None, refs=refs, extra=True)
    held = _run(mv, 0, p, 4, refs=refs, extra=True)
    assert held["slots"] == 4
    _assert_same(full, held)


def test_slots_objective_equals_resident(gpu):
    nx, ny, nz = 516, 512, 11
    mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=191, dtype="f32", speed=0.7, rw_sigma=0.4)
    p = api.verify_params(api.Params(CCPeakSearchDim=64), nz)
    s = np.random.default_rng(2).uniform(-1.5, 1.5, (nz, 2))
    res = []
    for slots in (None, 4, 7):
        with api.Plan(p, nx, ny, nz, 2, spectrum_slots=slots) as pl:
            pl.load_frames(mv.frames)
            pl.forward()
            res.append(pl.objective(s))
    for J, g, h in res[1:]:
        assert J == res[0][0]
        np.testing.assert_array_equal(g, res[0][1])
        np.testing.assert_array_equal(h, res[0][2])


def test_slots_rules(gpu):
    nx, ny, nz = 530, 520, 8
    mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=201, dtype="u8")
    p = api.verify_params(api.Params(crop_nsam=512, CCPeakSearchDim=64), nz)
    with pytest.raises(_lib.McError) as e:
        api.Plan(p, nx, ny, nz, 0, spectrum_slots=3)
    assert e.value.code == -1
    with api.Plan(p, nx, ny, nz, 0, spectrum_slots=4) as pl:
        pl.load_frames(mv.frames)
        pl.run()
        with pytest.raises(_lib.McError) as e:
            pl.fsc()
        assert e.value.code == -5 and "spectrum slots" in str(e.value)
    # as many slots as frames: the resident plan
    with api.Plan(p, nx, ny, nz, 0, spectrum_slots=nz) as pl:
        assert pl.spectrum_slots == 0


def _spec_bytes(n):
    return (n // 2 + 1) * ((n + 3) // 4 * 4) * 8


def test_automatic_slots_under_a_device_budget(gpu):
    nx, ny, nz = 530, 520, 12
    mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=211, dtype="u8", speed=0.6, rw_sigma=0.4)
    p = api.verify_params(api.Params(crop_nsam=512, CCPeakSearchDim=64, iter=1), nz)
    full = _run(mv, 0, p, None)
    L = _lib.lib()
    try:
        L.mc_debug_device_budget(KEEP_FREE + int(6.5 * _spec_bytes(512)))
        held = _run(mv, 0, p, None)
        assert held["slots"] == 6 and held["recomputes"] > 0
        _assert_same(full, held)
        L.mc_debug_device_budget(KEEP_FREE + 3 * _spec_bytes(512))
        with pytest.raises(_lib.McError) as e:
            api.Plan(p, nx, ny, nz, 0)
        assert e.value.code == -3
    finally:
        L.mc_debug_device_budget(0)


def test_batch_lanes_with_slot_plans(gpu):
    movies, ref = [], []
    for k, (nx, ny, nz) in enumerate([(530, 520, 10), (530, 520, 12), (300, 290, 9)]):
        mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=221 + k, dtype="u8", speed=0.6, rw_sigma=0.4)
        p = api.verify_params(api.Params(CCPeakSearchDim=64, iter=1), nz)
        ref.append(api.align(mv.frames, 0, p))
        movies.append({"params": p, "nx": nx, "ny": ny, "nz": nz, "mode": 0, "frames": mv.frames,
                       "image": np.empty_like(ref[-1]["image"]),
                       "frame_shifts": np.empty_like(ref[-1]["frame_shifts"])})
    L = _lib.lib()
    try:
        L.mc_debug_device_budget(KEEP_FREE + int(5.5 * _spec_bytes(512)))
        with api.Batch(0, lanes=2) as bt:
            res = bt.run(movies)
    finally:
        L.mc_debug_device_budget(0)
    assert all(r["status"] == 0 for r in res)
    for m, g in zip(movies, ref):
        np.testing.assert_array_equal(m["image"], g["image"])
        np.testing.assert_array_equal(m["frame_shifts"], g["frame_shifts"])


def test_single_graph_batch_rejects_slot_plans(gpu):
    """The one-graph batch needs every spectrum of a movie in HBM: under a
    device budget that forces spectrum slots it reports so, and runs again
    once the budget is lifted."""
    import torch
    mv = synth.make_movie(530, 520, 12, mean=2.0, seed=241, dtype="u8", speed=0.6, rw_sigma=0.4)
    p = api.verify_params(api.Params(crop_nsam=512, CCPeakSearchDim=64), 12)
    d = torch.from_numpy(np.ascontiguousarray(mv.frames)).cuda()
    img = torch.zeros((512, 512), dtype=torch.float32, pin_memory=True)
    movie = {"params": p, "nx": 530, "ny": 520, "nz": 12, "mode": 0, "device_ptr": d.data_ptr(),
             "image": img.numpy(), "frame_shifts": np.zeros((12, 2))}
    L = _lib.lib()
    try:
        L.mc_debug_device_budget(KEEP_FREE + int(5.5 * _spec_bytes(512)))
        with api.Batch(0, lanes=1, graph=True) as bt:
            res = bt.run([movie], check=False)
    finally:
        L.mc_debug_device_budget(0)
    assert res[0]["status"] == -5 and "spectrum slots" in res[0]["message"], res[0]
    with api.Batch(0, lanes=1, graph=True) as bt:
        res = bt.run([movie])
    assert res[0]["status"] == 0
    ref = api.align(mv.frames, 0, p)
    np.testing.assert_array_equal(img.numpy(), ref["image"])


@pytest.mark.slow
def test_c4_with_sixteen_slots_equals_resident(gpu):
    """The c4 movie (60 x 4096^2 float32, -itr 3, -ref 1) with 16 of its 60
    spectra held: the recomputing path gives the resident plan's shifts and
    sum bit for bit; its time against the resident run is printed."""
    import time
    import torch
    w = dict(synth.WORKLOADS["c4"])
    flags = dict(w.pop("flags"))
    frames, _ = synth.make_movie_torch(w["nx"], w["ny"], w["nframes"], mean=w["mean"], seed=0, dtype=w["dtype"],
                                       kind=w["kind"], speed=w.get("speed", 0.4), rw_sigma=w.get("rw_sigma", 0.3),
                                       amp=w.get("amp", 1.5), period=w.get("period", 20.0), device="cuda")
    nz, ny, nx = frames.shape
    p = api.verify_params(api.Params(**flags, refine=1), nz)
    out = {}
    for slots in (None, 16):
        with api.Plan(p, nx, ny, nz, 2, spectrum_slots=slots) as pl:
            pl.load_frames_device(frames.data_ptr(), 0, nz)
            pl.run()                                   # warm-up
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            img = pl.run()
            dt = time.perf_counter() - t0
            out[slots] = (img, pl.frame_shifts(), dt, pl.forward_recomputes, pl.info["device_bytes"])
    (i0, s0, t0, _, b0), (i1, s1, t1, r1, b1) = out[None], out[16]
    print(f"c4 -ref 1: resident {t0 * 1e3:.1f} ms, {b0 / 2**30:.2f} GiB; 16 slots {t1 * 1e3:.1f} ms "
          f"({t1 / t0:.2f}x), {b1 / 2**30:.2f} GiB, {r1} forward transforms recomputed over two runs")
    np.testing.assert_array_equal(s0, s1)
    np.testing.assert_array_equal(i0, i1)
    assert b1 < b0


def test_short_movies_stay_resident(gpu):
    """Fewer frames than the smallest slot count: every spectrum resident."""
    mv = synth.make_movie(300, 290, 3, mean=2.0, seed=231, dtype="u8")
    p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=0), 3)
    with api.Plan(p, 300, 290, 3, 0) as pl:
        assert pl.spectrum_slots == 0
        pl.load_frames(mv.frames)
        pl.run()
