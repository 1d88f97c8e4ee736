"""mc_pair_window_static: the allocation-free entry point.

It exists for callers that must not allocate device memory (an acquisition
or streaming loop that owns a fixed memory budget, a framework that forbids
allocation after setting up its pool).  This file is collected last, runs in
a fresh process or after the other tests, and checks two calls in a row
through the C ABI against the CC windows of the regular plan path
(mc_plan_pairs / mc_plan_get_boxes) at the tolerance the parity tests use:
at n = 512 (the runtime-split register kernel), n = 2048 and 4096 (compiled
splits), an odd window (pbx 95) and the limit case n = 4096, pbx = 128 that
lays out 4.2 MB of the 5 MiB scratch.  It also checks the defining property:
repeated calls leave the device's free memory unchanged.
"""
import ctypes as C

import numpy as np
import pytest

from motioncorr1exp_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu

WINDOW_RTOL = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(np.asarray(b, np.float64)))


def _plan_windows(n, box, nz=6):
    mv = synth.make_movie(n + 8, n, nz, mean=1.5, seed=21 + n + box, dtype="f32", speed=0.6, rw_sigma=0.3)
    p = api.verify_params(api.Params(CCPeakSearchDim=box, FrameDistOffset=2), nz)
    with api.Plan(p, n + 8, n, nz, 2) as pl:
        pl.load_frames(mv.frames)
        pl.forward()
        pl.pairs()
        boxes = pl.boxes()
        pairs = pl.pair_results()["pairs"]
        spectra = {f: pl.spectrum(f) for f in range(nz)}   # (ky, kx) reference layout
        split = (pl.info["prune_p"], pl.info["prune_q"])
    return p, boxes, pairs, spectra, split


def _call(L, da, db, n, box, bfactor, out):
    return L.mc_pair_window_static(C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), n, n, box,
                                   C.c_float(bfactor), C.c_void_p(out.data_ptr()), None)


@pytest.mark.parametrize("n,box", [(512, 96), (1024, 95), (2048, 96), (4096, 128)])
def test_static_scratch_window_matches_plan(gpu, n, box):
    import torch
    p, boxes, pairs, spectra, split = _plan_windows(n, box)
    L = _lib.lib()
    h = n // 2 + 1
    out = torch.empty((box, box), dtype=torch.float32, device="cuda")
    for call, r in enumerate((0, len(pairs) - 1)):           # two calls in a row
        i, j = (int(v) for v in pairs[r])
        # library layout: spec[kx * ldn + ky], ldn = n
        da = torch.from_numpy(np.ascontiguousarray(spectra[i].T).view(np.float32)).cuda()
        db = torch.from_numpy(np.ascontiguousarray(spectra[j].T).view(np.float32)).cuda()
        assert da.numel() == 2 * h * n
        out.fill_(float("nan"))
        rc = _call(L, da, db, n, box, p.bfactor, out)
        assert rc == 0, L.mc_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert rel_l2(got, boxes[r]) <= WINDOW_RTOL, (n, box, split, call, rel_l2(got, boxes[r]))


def test_static_scratch_allocates_nothing(gpu):
    """After one warm-up call (kernel modules loaded), further calls change
    the device's free memory by nothing."""
    import torch
    n, box = 2048, 96
    p, boxes, pairs, spectra, _ = _plan_windows(n, box, nz=6)
    L = _lib.lib()
    i, j = (int(v) for v in pairs[0])
    da = torch.from_numpy(np.ascontiguousarray(spectra[i].T).view(np.float32)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(spectra[j].T).view(np.float32)).cuda()
    out = torch.empty((box, box), dtype=torch.float32, device="cuda")
    assert _call(L, da, db, n, box, p.bfactor, out) == 0, L.mc_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(8):
        assert _call(L, da, db, n, box, p.bfactor, out) == 0, L.mc_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert rel_l2(out.cpu().numpy(), boxes[0]) <= WINDOW_RTOL


def test_static_scratch_rejects_oversize(gpu):
    L = _lib.lib()
    rc = L.mc_pair_window_static(C.c_void_p(16), C.c_void_p(16), 8192, 8192, 96, C.c_float(150.0),
                                 C.c_void_p(16), None)
    assert rc == -4
    assert b"4096" in L.mc_last_error()
    rc = L.mc_pair_window_static(C.c_void_p(16), C.c_void_p(16), 512, 512, 200, C.c_float(150.0),
                                 C.c_void_p(16), None)
    assert rc == -4
