"""The device-only movie pipeline (device FP64 solve, one synchronisation,
CUDA-graph capture and replay) against the staged path with the host solve."""
import numpy as np
import pytest

from motioncorr1exp_b200 import api, synth

pytestmark = pytest.mark.gpu


def _staged(pl):
    lines = []
    pl.set_log(lines.append)
    pl.forward()
    pl.pairs()
    pl.solve()
    pl.iterate()
    img = pl.sum()
    return img, pl.frame_shifts().copy(), pl.pair_results(), pl.ki(), "".join(lines)


def _device(pl, frames):
    lines = []
    pl.set_log(lines.append)
    pl.load_frames(frames)
    img = pl.run()
    return img, pl.frame_shifts().copy(), pl.pair_results(), pl.ki(), "".join(lines)


@pytest.mark.parametrize("kw", [dict(), dict(bAlignToMid=0, nStartSum=2), dict(kiThresh=0.05, FrameDistOffset=1)])
def test_device_pipeline_matches_staged(gpu, kw):
    mv = synth.make_movie(300, 290, 12, mean=2.0, seed=31, dtype="u8", speed=0.6, rw_sigma=0.5)
    p = api.verify_params(api.Params(**kw), 12)
    with api.Plan(p, 300, 290, 12, 0) as pl:
        pl.load_frames(mv.frames)
        img_s, fs_s, pr_s, ki_s, log_s = _staged(pl)
        img_d, fs_d, pr_d, ki_d, log_d = _device(pl, mv.frames)      # captures the graph
        img_r, fs_r, pr_r, ki_r, log_r = _device(pl, mv.frames)      # replays it
    for k in ("pairs", "shift", "cc", "peak"):
        np.testing.assert_array_equal(pr_s[k], pr_d[k])
        np.testing.assert_array_equal(pr_d[k], pr_r[k])
    np.testing.assert_array_equal(ki_s["kept"], ki_d["kept"])
    np.testing.assert_allclose(ki_s["ki1"], ki_d["ki1"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(fs_s, fs_d, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(fs_d, fs_r)
    np.testing.assert_allclose(img_d, img_s, rtol=0, atol=1e-6 * np.abs(img_s).max())
    np.testing.assert_array_equal(img_d, img_r)
    # identical text apart from the header lines the run path adds
    body_d = log_d[log_d.index("\nRead stack:"):]
    assert body_d == log_s[log_s.index("\nRead stack:"):]


def test_run_host_device_path(gpu):
    mv = synth.make_movie(256, 256, 10, mean=2.0, seed=32, dtype="u8", speed=0.5, rw_sigma=0.4)
    p = api.verify_params(api.Params(CCPeakSearchDim=64), 10)
    with api.Plan(p, 256, 256, 10, 0) as pl:
        img_h = pl.run_host(mv.frames)
        fs_h = pl.frame_shifts().copy()
        pl.load_frames(mv.frames)
        img_r = pl.run()
        np.testing.assert_array_equal(img_h, img_r)
        np.testing.assert_array_equal(fs_h, pl.frame_shifts())
