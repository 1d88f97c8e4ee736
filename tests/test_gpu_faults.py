"""Failure paths, injected on the host (no GPU fault): every device or pinned
allocation a plan makes is failed in turn through mc_debug_fail_alloc; the
creation reports MC_E_NOMEM, releases what it had allocated and leaves the
device usable, and a batch whose second movie cannot get its plan reports
that movie's status while the others complete."""
import numpy as np
import pytest

from motioncorr1exp_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu


def _count_allocs(p, nx, ny, nz, mode):
    """Allocations of one plan creation: the first countdown that succeeds."""
    L = _lib.lib()
    k = 1
    try:
        while True:
            L.mc_debug_fail_alloc(k)
            try:
                pl = api.Plan(p, nx, ny, nz, mode)
            except _lib.McError as e:
                assert e.code == -3 and "injected" in str(e), str(e)
                k += 1
                assert k < 500
                continue
            pl.close()
            return k - 1
    finally:
        L.mc_debug_fail_alloc(0)


def test_every_plan_allocation_failure_is_clean(gpu):
    import torch
    mv = synth.make_movie(300, 290, 8, mean=1.5, seed=91, dtype="u8")
    p = api.verify_params(api.Params(CCPeakSearchDim=64), 8)
    ref = api.align(mv.frames, 0, p)           # warm-up: modules loaded, reference result
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    n = _count_allocs(p, 300, 290, 8, 0)
    assert n >= 20                              # buffers, tables, pinned staging
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert abs(free0 - free1) <= 4 << 20, (free0, free1)   # nothing leaked by the failed creations
    got = api.align(mv.frames, 0, p)           # and the device still works
    np.testing.assert_array_equal(got["image"], ref["image"])
    np.testing.assert_array_equal(got["frame_shifts"], ref["frame_shifts"])


def test_batch_reports_the_movie_whose_plan_failed(gpu):
    a = synth.make_movie(256, 256, 8, mean=1.5, seed=92, dtype="u8")
    b = synth.make_movie(300, 290, 8, mean=1.5, seed=93, dtype="u8")
    p = api.verify_params(api.Params(CCPeakSearchDim=64), 8)
    na = _count_allocs(p, 256, 256, 8, 0)
    L = _lib.lib()
    movies = [{"params": p, "nx": 256, "ny": 256, "nz": 8, "mode": 0, "frames": a.frames},
              {"params": p, "nx": 300, "ny": 290, "nz": 8, "mode": 0, "frames": b.frames},
              {"params": p, "nx": 256, "ny": 256, "nz": 8, "mode": 0, "frames": a.frames}]
    with api.Batch(0, lanes=1) as bt:
        L.mc_debug_fail_alloc(na + 1)           # the first allocation of the second movie's plan
        try:
            res = bt.run(movies, check=False)
        finally:
            L.mc_debug_fail_alloc(0)
        assert [r["status"] for r in res] == [0, -3, 0]
        assert "injected" in res[1]["message"]
        res = bt.run(movies)                     # the runner recovers on the next batch
        assert all(r["status"] == 0 for r in res)
