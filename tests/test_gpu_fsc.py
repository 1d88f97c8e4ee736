"""-fsc (PlotFSC, DFAlign.cu:212-326) through the C ABI against the FP64
oracle: the four FSC curves per shell from even/odd halves of the summed
frames.  Shell membership and the along/across split use the reference's
float r and angle in both; the shell sums are FP32 spectra products summed
in FP64 on the GPU vs FP64 throughout in the oracle, so each FSC value is
within 1e-4 (absolute)."""
import numpy as np
import pytest

from motioncorr1exp_b200 import _lib, api, synth
from oracle import mc_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("geom,kw", [
    ((520, 512, 8), dict()),
    ((520, 512, 9), dict(bAlignToMid=0, nStartSum=1, nEndSum=7)),
    ((900, 880, 6), dict(FrameDistOffset=1)),
    ((1040, 1030, 6), dict(bin=2.0, FrameDistOffset=1)),
])
def test_fsc_matches_oracle(gpu, geom, kw):
    nx, ny, nz = geom
    mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=81 + nz, dtype="u8", speed=0.9, rw_sigma=0.4)
    kw = {"CCPeakSearchDim": 64, "FrameDistOffset": 2, **kw}
    p = api.verify_params(api.Params(**kw), nz)
    with api.Plan(p, nx, ny, nz, 0) as pl:
        pl.load_frames(mv.frames)
        pl.run()
        got = pl.fsc()
        nu, n = pl.info["nsam_unbin"], pl.nsam
        F = [O.forward_spectrum(O.decode_frame(mv.frames[f], 0), 0, 0, nu, n) for f in range(nz)]
        sh, first, last = pl.sum_shifts()
        drift = pl.frame_shifts()[last]
    want = O.fsc_table(F, first, last, sh, bool(p.bAlignToMid), drift)
    assert got.shape == want.shape == ((n // 2 + 1) // (n // 400) + 1, 5)
    np.testing.assert_array_equal(got[:, 0], want[:, 0])
    assert np.abs(got[:, 1:] - want[:, 1:]).max() < 1e-4
    assert np.count_nonzero(want[:, 1:]) > 0.9 * want[:, 1:].size


def test_fsc_needs_400(gpu):
    mv = synth.make_movie(300, 292, 6, mean=2.0, seed=85, dtype="u8")
    p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=1), 6)
    with api.Plan(p, 300, 292, 6, 0) as pl:
        pl.load_frames(mv.frames)
        pl.run()
        with pytest.raises(_lib.McError) as ei:
            pl.fsc()
        assert ei.value.code == -4
