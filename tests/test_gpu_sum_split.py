"""The image sum of two-level sizes runs as two kernels (k_shift_acc, then
k_sum_cols2l with a transposed store); MC_SUM_FUSED=1 at plan creation keeps
the single fused kernel.  Both add the same products in the same frame order
and run the same transform per column, so the images agree bit for bit.  The
raw and partial sums (accumulation only) are compared the same way."""
import os

import numpy as np
import pytest

from motioncorr1exp_b200 import api, synth

pytestmark = pytest.mark.gpu


def _run(mv, p, nx, ny, nz, fused):
    old = os.environ.pop("MC_SUM_FUSED", None)
    if fused:
        os.environ["MC_SUM_FUSED"] = "1"
    try:
        with api.Plan(p, nx, ny, nz, 0) as pl:
            pl.load_frames(mv.frames[pl.info["nstart"]: pl.info["nend"] + 1])
            img = pl.run()
            _, first, last = pl.sum_shifts()
            raw = pl.raw_sum()
            part = pl.sum_to(first + (last - first) // 2 + pl.info["nstart"])
            return img, raw, part
    finally:
        os.environ.pop("MC_SUM_FUSED", None)
        if old is not None:
            os.environ["MC_SUM_FUSED"] = old


@pytest.mark.parametrize("crop, nx, ny", [(512, 560, 540), (1024, 1060, 1040)])
def test_split_sum_equals_fused(gpu, crop, nx, ny):
    nz = 10
    mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=83, dtype="u8", speed=0.6, rw_sigma=0.4)
    p = api.verify_params(api.Params(crop_nsam=crop, CCPeakSearchDim=64), nz)
    split = _run(mv, p, nx, ny, nz, fused=False)
    fused = _run(mv, p, nx, ny, nz, fused=True)
    assert split[0].shape == (crop, crop)
    for a, b in zip(split, fused):
        assert np.array_equal(a, b)
