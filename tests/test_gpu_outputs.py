"""Extra sum-stage outputs (-srs raw sum, -2es second sum, -ssc corrected
frames) and the exact count sums, through the C ABI against the FP64 oracle.

Tolerances: images relative L2 <= 1e-5 (FP32 transforms vs FP64); count
sums bit-exact."""
import numpy as np
import pytest

from motioncorr1exp_b200 import api, synth
from oracle import mc_oracle as O

pytestmark = pytest.mark.gpu

IMAGE_RTOL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _spectra(frames, mode, p, nu, n):
    return [O.forward_spectrum(O.decode_frame(frames[f], mode), p.crop_offsetx, p.crop_offsety, nu, n)
            for f in range(p.nStart, p.nEnd + 1)]


@pytest.mark.parametrize("kw", [dict(), dict(bAlignToMid=0, nStartSum=2, nEndSum=9), dict(bin=2.0, nStart=1)])
def test_raw_second_and_corrected(gpu, kw):
    nz = 12
    mv = synth.make_movie(300, 292, nz, mean=2.0, seed=61, dtype="u8", speed=0.6, rw_sigma=0.4)
    p = api.verify_params(api.Params(CCPeakSearchDim=64, **kw), nz)
    with api.Plan(p, 300, 292, nz, 0) as pl:
        pl.load_frames(mv.frames[pl.info["nstart"]: pl.info["nend"] + 1])
        img = pl.run()
        nu, n = pl.info["nsam_unbin"], pl.nsam
        F = _spectra(mv.frames, 0, p, nu, n)
        sh, first, last = pl.sum_shifts()
        # -srs: unaligned sum of nStartSum..nEndSum
        raw = pl.raw_sum()
        assert rel_l2(raw, O.raw_sum_image(F, first, last)) <= IMAGE_RTOL
        # -2es: the aligned prefix sum; up to nEndSum it is the corrected sum itself
        assert rel_l2(pl.sum_to(last + pl.info["nstart"]), img) <= 1e-6
        mid = first + (last - first) // 2
        part = pl.sum_to(mid + pl.info["nstart"])
        S = np.zeros_like(F[0])
        for k in range(first, mid + 1):
            apply = not (k == first and not p.bAlignToMid)
            S = S + (O.phase_shift(F[k], sh[k, 0], sh[k, 1]) if apply else F[k])
        assert rel_l2(part, O.spectrum_to_image(S)) <= IMAGE_RTOL
        # the reference's clamp: a last frame at or before the first summed one means "all frames"
        assert rel_l2(pl.sum_to(first + pl.info["nstart"]), img) <= 1e-6
        # -ssc: each aligned frame; together they add up to the corrected sum
        acc = np.zeros((n, n))
        for k in range(first, last + 1):
            fr = pl.corrected_frame(k + pl.info["nstart"])
            apply = not (k == first and not p.bAlignToMid)
            want = O.spectrum_to_image(O.phase_shift(F[k], sh[k, 0], sh[k, 1]) if apply else F[k])
            assert rel_l2(fr, want) <= IMAGE_RTOL
            acc += fr
        assert rel_l2(acc, img) <= IMAGE_RTOL
        with pytest.raises(Exception):
            pl.corrected_frame(last + pl.info["nstart"] + 1)


@pytest.mark.parametrize("mode,dtype", [(0, np.int8), (1, np.int16), (6, np.uint16), (api.MODE_U8, np.uint8)])
def test_count_sum_exact(gpu, mode, dtype):
    rng = np.random.default_rng(62 + mode)
    nz, ny, nx = 9, 203, 230
    lo, hi = {0: (-128, 128), 1: (-32768, 32768), 6: (0, 65536), api.MODE_U8: (0, 256)}[mode]
    frames = rng.integers(lo, hi, size=(nz, ny, nx)).astype(dtype)
    p = api.verify_params(api.Params(CCPeakSearchDim=32, crop_offsetx=5, crop_offsety=3, nStartSum=1,
                                     nEndSum=7, FrameDistOffset=1), nz)
    with api.Plan(p, nx, ny, nz, mode) as pl:
        pl.load_frames(frames)
        got = pl.count_sum()
        nu = pl.info["nsam_unbin"]
        want = O.count_sum(frames, mode, 5, 3, nu, 1, 7)
        np.testing.assert_array_equal(got.astype(np.int64), want)


def test_count_sum_bound_frames_and_float_rejected(gpu):
    import torch
    mv = synth.make_movie(256, 256, 6, mean=1.5, seed=63, dtype="u8")
    p = api.verify_params(api.Params(CCPeakSearchDim=32, FrameDistOffset=1), 6)
    d = torch.from_numpy(mv.frames).cuda()
    with api.Plan(p, 256, 256, 6, 0) as pl:
        pl.bind_frames_device(d.data_ptr())
        np.testing.assert_array_equal(pl.count_sum().astype(np.int64),
                                      O.count_sum(mv.frames, 0, 0, 0, 256, 0, 5))
    f32 = synth.make_movie(128, 128, 6, mean=1.5, seed=64, dtype="f32")
    with api.Plan(p, 128, 128, 6, 2) as pl:
        pl.load_frames(f32.frames)
        with pytest.raises(Exception):
            pl.count_sum()


@pytest.mark.parametrize("kw", [dict(), dict(bin=2.0)])
def test_unsigned_bytes_equal_uint16(gpu, kw):
    """MC_MODE_U8 (8-bit TIFF words) decodes bytes above 127 as unsigned: the
    same movie as uint16 (mode 6) gives bit-identical results; mode 0 reads
    the same bytes as signed char and differs."""
    rng = np.random.default_rng(65)
    base = synth.make_movie(300, 292, 8, mean=2.0, seed=66, dtype="u8", speed=0.6, rw_sigma=0.4).frames
    frames = (base.astype(np.int32) + rng.integers(100, 140, base.shape)).clip(0, 255).astype(np.uint8)
    assert frames.max() > 127
    p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=2, **kw), 8)
    r8 = api.align(frames, api.MODE_U8, p)
    r16 = api.align(frames.astype(np.uint16), 6, p)
    np.testing.assert_array_equal(r8["image"], r16["image"])
    np.testing.assert_array_equal(r8["frame_shifts"], r16["frame_shifts"])
    rs = api.align(frames.view(np.int8), 0, p)
    assert not np.array_equal(rs["image"], r8["image"])


@pytest.mark.parametrize("kw", [dict(), dict(crop_offsetx=6, crop_nsam=256, bin=2.0)])
def test_half_frames(gpu, kw):
    """MC_MODE_F16 (MRC2014 mode 12): integer counts stored as IEEE half give
    results bit-identical to the same counts as float32 (the widening is
    exact), on every forward path (two-level raw rows, -bin 2 split, the
    generic engine); non-integer frames stored as half match the FP64
    oracle run on the same half values."""
    mv = synth.make_movie(300, 292, 8, mean=2.0, seed=67, dtype="f32", speed=0.6, rw_sigma=0.4)
    assert mv.frames.max() < 2048
    p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=2, **kw), 8)
    r32 = api.align(mv.frames, 2, p)
    r16 = api.align(mv.frames.astype(np.float16), api.MODE_F16, p)
    np.testing.assert_array_equal(r16["image"], r32["image"])
    np.testing.assert_array_equal(r16["frame_shifts"], r32["frame_shifts"])
    # non-integer pixels: the half values are what the oracle decodes
    fr = (mv.frames * np.float32(1.37) + np.float32(0.25)).astype(np.float16)
    g = api.align(fr, api.MODE_F16, p)
    ref = O.align_movie(fr, api.MODE_F16, O.Params(**{k: getattr(p, k) for k in O.Params.__dataclass_fields__}))
    fo = np.stack([ref.frame_shift.real, ref.frame_shift.imag], 1)
    assert np.max(np.abs(g["frame_shifts"] - fo)) <= 0.01
    assert np.linalg.norm(g["image"] - ref.image) / np.linalg.norm(ref.image) <= 1e-5
