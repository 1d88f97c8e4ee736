"""Adjoint of the phase-shift-and-sum and the gradient refinement (added
method; no reference counterpart).

  * objective, gradient and Hessian blocks vs the FP64 oracle
    (relative 1e-5 on J, 1e-4 of the largest entry on gradient/Hessian);
  * adjoint gradient vs central finite differences of the CUDA objective,
    h = 1e-3 px (relative 2e-3 of the gradient scale);
  * the torch.autograd.Function harness returns the adjoint gradient;
  * refined shifts have a lower ground-truth RMSE than the plain peak fit.
"""
import numpy as np
import pytest

from motioncorr1exp_b200 import api, synth
from oracle import mc_oracle as O

pytestmark = pytest.mark.gpu


def _plan(n=256, nframes=6, seed=3, **kw):
    mv = synth.make_movie(n + 4, n, nframes, mean=2.0, seed=seed, dtype="f32", speed=0.7, rw_sigma=0.4)
    p = api.verify_params(api.Params(CCPeakSearchDim=64, **kw), nframes)
    pl = api.Plan(p, n + 4, n, nframes, 2)
    pl.load_frames(mv.frames)
    pl.forward()
    return pl, mv, p


def test_objective_matches_fp64_oracle(gpu):
    pl, mv, p = _plan()
    with pl:
        rng = np.random.default_rng(0)
        s = rng.uniform(-1.5, 1.5, (pl.nframe, 2))
        J, g, h = pl.objective(s)
        F = [O.forward_spectrum(O.decode_frame(mv.frames[k], 2), 0, 0, pl.nsam, pl.nsam) for k in range(pl.nframe)]
        Jo, go, ho = O.sum_objective(F, s, p.bfactor)
    assert abs(J - Jo) <= 1e-5 * abs(Jo)
    np.testing.assert_allclose(g, go, atol=1e-4 * np.abs(go).max())
    np.testing.assert_allclose(h, ho, atol=1e-4 * np.abs(ho).max())


def test_adjoint_vs_central_differences(gpu):
    pl, mv, p = _plan(seed=5)
    with pl:
        rng = np.random.default_rng(1)
        s = rng.uniform(-1.0, 1.0, (pl.nframe, 2))
        _, g, _ = pl.objective(s)
        hstep = 1e-3
        scale = np.abs(g).max()
        for k in (0, 2, pl.nframe - 1):
            for c in (0, 1):
                sp, sm = s.copy(), s.copy()
                sp[k, c] += hstep
                sm[k, c] -= hstep
                fd = (pl.objective(sp)[0] - pl.objective(sm)[0]) / (2 * hstep)
                assert abs(fd - g[k, c]) <= 2e-3 * scale, (k, c, fd, g[k, c])


def test_torch_autograd_function(gpu):
    import torch
    from motioncorr1exp_b200.autograd import sum_objective
    pl, mv, p = _plan(seed=7)
    with pl:
        s = torch.tensor(np.random.default_rng(2).uniform(-1, 1, (pl.nframe, 2)), dtype=torch.float64,
                         requires_grad=True)
        J = sum_objective(s, pl)
        J.backward()
        _, g, _ = pl.objective(s.detach().numpy())
        np.testing.assert_allclose(s.grad.numpy(), g, rtol=1e-12, atol=0)
        assert float(J.detach()) == pytest.approx(pl.objective(s.detach().numpy())[0], rel=1e-12)


def _truth_rmse(shifts, truth):
    d = shifts + (truth - truth[0])
    d = d - d.mean(axis=0)   # a common offset does not change the aligned sum
    return float(np.sqrt(np.mean(np.sum(d * d, axis=1))))


def test_refinement_lowers_truth_rmse(gpu):
    plain, refined = [], []
    for seed in (11, 12, 13):
        mv = synth.make_movie(512, 512, 20, mean=1.0, seed=seed, dtype="f32", kind="jitter", rw_sigma=0.8,
                              amp=1.5, period=20.0)
        for ref, acc in ((0, plain), (1, refined)):
            p = api.verify_params(api.Params(iter=2, iterthres=0.001, refine=ref), 20)
            res = api.align(mv.frames, 2, p)
            acc.append(_truth_rmse(res["frame_shifts"], mv.truth))
    assert np.mean(refined) < np.mean(plain), (plain, refined)


def test_refine_keeps_reference_frame_and_logs(gpu):
    pl, mv, p = _plan(n=256, nframes=8, seed=9)
    lines = []
    with pl:
        pl.set_log(lines.append)
        pl.pairs()
        pl.solve()
        pl.iterate()
        before = pl.frame_shifts().copy()
        pl.refine(4)
        after = pl.frame_shifts()
    assert after[0].tolist() == [0.0, 0.0]
    assert np.max(np.abs(after - before)) < 0.5
    assert any("Gradient refinement" in l for l in lines)


@pytest.mark.slow
def test_adjoint_at_4096(gpu):
    """c4's frame size (4096^2 float32, counts of mean 1.0, the c4 drift
    model) with 6 frames: the adjoint gradient against central finite
    differences of the CUDA objective (h = 1e-3 px) and against the FP64
    oracle's gradient and Hessian blocks."""
    import torch
    n, nf = 4096, 6
    frames, _ = synth.make_movie_torch(n, n, nf, mean=1.0, seed=21, dtype="f32", kind="jitter", rw_sigma=0.8,
                                       amp=1.5, period=20.0, device="cuda")
    host = frames.cpu().numpy()
    p = api.verify_params(api.Params(CCPeakSearchDim=96), nf)
    with api.Plan(p, n, n, nf, 2) as pl:
        pl.load_frames_device(frames.data_ptr(), 0, nf)
        pl.forward()
        torch.cuda.synchronize()
        s = np.random.default_rng(4).uniform(-1.5, 1.5, (nf, 2))
        J, g, h = pl.objective(s)
        scale = np.abs(g).max()
        for k in (0, nf // 2, nf - 1):
            for c in (0, 1):
                sp, sm = s.copy(), s.copy()
                sp[k, c] += 1e-3
                sm[k, c] -= 1e-3
                fd = (pl.objective(sp)[0] - pl.objective(sm)[0]) / 2e-3
                assert abs(fd - g[k, c]) <= 2e-3 * scale, (k, c, fd, g[k, c])
    F = [O.forward_spectrum(O.decode_frame(host[k], 2), 0, 0, n, n) for k in range(nf)]
    Jo, go, ho = O.sum_objective(F, s, p.bfactor)
    assert abs(J - Jo) <= 1e-5 * abs(Jo)
    np.testing.assert_allclose(g, go, atol=1e-4 * np.abs(go).max())
    np.testing.assert_allclose(h, ho, atol=1e-4 * np.abs(ho).max())
