"""Parity of the CUDA path (through the C ABI of libmc.so) with the FP64 oracle.

Tolerances (the correctness bar of this path):
  * integer box peaks: bit-exact, except a near-tie where the oracle's own CC
    values at the two positions agree within 1e-5 (relative) -- FP32
    transforms cannot order them; that pair's shift then within 2/32 px;
  * pair shifts (1/32-px grid): equal, except a documented near-tie where the
    oracle's own upsampled map differs by < 1e-5 (relative) between the two
    neighbouring grid points;
  * per-frame shifts: within 0.01 px of the oracle;
  * summed image: relative L2 <= 1e-5;
  * spectra: relative L2 <= 1e-5 (FP32 transforms vs FP64).
"""
import numpy as np
import pytest

from motioncorr1exp_b200 import api, synth
from oracle import mc_oracle as O

pytestmark = pytest.mark.gpu

SHIFT_TOL = 0.01
IMAGE_RTOL = 1e-5
SPEC_RTOL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def to_oparams(p: api.Params) -> O.Params:
    return O.Params(**{k: getattr(p, k) for k in O.Params.__dataclass_fields__})


def run_both(frames, mode, params, refs=None, nz=None, stretch=None):
    nz = nz if nz is not None else frames.shape[0]
    p = api.verify_params(params, nz)
    g = api.align(frames, mode, p, nz=nz, refs=refs, stretch=stretch)
    ref = O.align_movie(frames, mode, to_oparams(p), nz_file=nz, refs=refs, stretch=stretch or (1.0, 1.0))
    return g, ref, p


def near_tie(box_map, n, nps, sx_o, sy_o, sx_g, sy_g):
    """True when the GPU's pair shift differs from the oracle's by one grid
    step at a point where the oracle's own upsampled map is flat to 1e-5."""
    if max(abs(sx_o - sx_g), abs(sy_o - sy_g)) > 1.5 / 32:
        return False
    box = box_map.shape[0]
    ix, iy = O.integer_peak(box_map, nps)
    offx = min(max(ix - 8, 0), box - 16)
    offy = min(max(iy - 8, 0), box - 16)
    f = O.upsampled_subbox(box_map, offx, offy)

    def val(sx, sy):
        X = int(round((sx + box // 2 - offx) * 32))
        Y = int(round((sy + box // 2 - offy) * 32))
        return f[Y % 512, X % 512]
    a, b = val(sx_o, sy_o), val(sx_g, sy_g)
    return abs(a - b) <= 1e-5 * abs(a)


def check_pairs(g, ref, n, nps, boxes_o=None):
    assert np.array_equal(g["pairs"], np.array(ref.pairs, dtype=np.int32))
    so = np.stack([ref.pair_shift.real, ref.pair_shift.imag], 1)
    sg = g["shift"].astype(np.float64)
    peak_ties = np.nonzero(np.any(g["peak"] != ref.pair_peak, axis=1))[0]
    for r in peak_ties:
        assert boxes_o is not None, f"pair {r}: peak {g['peak'][r]} vs {ref.pair_peak[r]}"
        (gx, gy), (ox, oy) = g["peak"][r], ref.pair_peak[r]
        vo, vg = boxes_o[r][oy, ox], boxes_o[r][gy, gx]
        assert abs(vo - vg) <= 1e-5 * abs(vo), f"pair {r}: peak {g['peak'][r]} vs {ref.pair_peak[r]}"
        assert np.max(np.abs(so[r] - sg[r])) <= 2.0 / 32 + 1e-9, f"pair {r}: {sg[r]} vs {so[r]}"
    assert len(peak_ties) <= max(1, len(ref.pairs) // 50)
    bad = [r for r in np.nonzero(np.any(so != sg, axis=1))[0] if r not in set(peak_ties)]
    for r in bad:
        assert boxes_o is not None, f"pair {r}: {sg[r]} vs {so[r]}"
        assert near_tie(boxes_o[r], n, nps, so[r, 0], so[r, 1], sg[r, 0], sg[r, 1]), \
            f"pair {r}: {sg[r]} vs {so[r]}"
    assert len(bad) <= max(1, len(ref.pairs) // 50)
    np.testing.assert_allclose(g["cc"], ref.pair_cc, rtol=1e-4)


def oracle_boxes(frames, mode, p, refs=None):
    nz, ny, nx = frames.shape
    nu = O.verify_crop_size(nx, ny, p.crop_offsetx, p.crop_offsety, p.crop_nsam, p.bin)
    n = O.binned_size(nu, p.bin)
    nf = p.nEnd - p.nStart + 1
    refs = refs or {}
    Fa, Fb = [], []
    for f in range(p.nStart, p.nEnd + 1):
        a, b = O.apply_refs(O.decode_frame(frames[f], mode), refs.get("dark"), refs.get("dark2"),
                            refs.get("norm"), refs.get("norm2"))
        Fa.append(O.forward_spectrum(a, p.crop_offsetx, p.crop_offsety, nu, n))
        Fb.append(O.forward_spectrum(b, p.crop_offsetx, p.crop_offsety, nu, n))
    mask = O.bfactor_mask(n, p.bfactor)
    return np.stack([O.cc_box(O.cc_map(Fa[i], Fb[j], mask, n), n, p.CCPeakSearchDim)
                     for i, j in O.pair_list(nf, p.FrameDistOffset)]), Fa, Fb


# ----------------------------------------------------------------- engine --
@pytest.mark.parametrize("n", [2, 3, 4, 5, 7, 8, 11, 13, 16, 17, 53, 64, 70, 106, 202, 210, 1024, 1855,
                               3710, 4096, 7420])
def test_fft_engine(gpu, n):
    import torch
    rng = np.random.default_rng(n)
    x = (rng.standard_normal((3, n)) + 1j * rng.standard_normal((3, n))).astype(np.complex64)
    d_in = torch.from_numpy(x.view(np.float32)).cuda()
    d_out = torch.empty_like(d_in)
    for inv in (False, True):
        api.fft1d(d_in.data_ptr(), d_out.data_ptr(), n, 3, inv)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(np.complex64).astype(np.complex128)
        ref = np.fft.ifft(x.astype(np.complex128), axis=1) * n if inv else np.fft.fft(x.astype(np.complex128), axis=1)
        assert rel_l2(got, ref) < 2e-6, (n, inv, rel_l2(got, ref))


# ---------------------------------------------------------------- forward --
@pytest.mark.parametrize("nx,ny,mode,offx,offy,crd,bin_", [
    (180, 170, 2, 0, 0, 0, 1.0),
    (256, 256, 0, 0, 0, 0, 1.0),
    (300, 260, 1, 10, 4, 0, 1.0),
    (424, 430, 6, 0, 0, 0, 2.0),
    (260, 250, 2, 3, 5, 200, 1.0),
    (300, 300, 2, 0, 0, 0, 1.5),
    # -bin 2 from 2N with a two-level N: the radix-2 split kernels (raw staging
    # of every pixel type, unaligned crop rows)
    (520, 512, 0, 0, 0, 0, 2.0),
    (512, 530, 1, 0, 0, 0, 2.0),
    (515, 520, 6, 3, 0, 0, 2.0),
    (2060, 2050, 2, 5, 1, 2048, 2.0),
])
def test_forward_matches_oracle(gpu, nx, ny, mode, offx, offy, crd, bin_):
    rng = np.random.default_rng(nx + ny)
    nz = 3
    if mode == 0:
        frames = rng.integers(0, 120, (nz, ny, nx)).astype(np.uint8)
    elif mode == 1:
        frames = rng.integers(-3000, 3000, (nz, ny, nx)).astype(np.int16)
    elif mode == 6:
        frames = rng.integers(0, 60000, (nz, ny, nx)).astype(np.uint16)
    else:
        frames = rng.normal(5, 2, (nz, ny, nx)).astype(np.float32)
    p = api.verify_params(api.Params(crop_offsetx=offx, crop_offsety=offy, crop_nsam=crd, bin=bin_,
                                      FrameDistOffset=0), nz)
    with api.Plan(p, nx, ny, nz, mode) as pl:
        pl.load_frames(frames)
        pl.forward()
        nu = O.verify_crop_size(nx, ny, offx, offy, crd, bin_)
        n = O.binned_size(nu, bin_)
        assert (pl.info["nsam_unbin"], pl.nsam) == (nu, n)
        for f in range(nz):
            ref = O.forward_spectrum(O.decode_frame(frames[f], mode), offx, offy, nu, n)
            got = pl.spectrum(f)
            assert rel_l2(got, ref) < SPEC_RTOL
        np.testing.assert_allclose(pl.frame_means(), [O.forward_spectrum(
            O.decode_frame(frames[f], mode), offx, offy, nu, n)[0, 0].real / n / n for f in range(nz)], rtol=1e-5)


@pytest.mark.parametrize("two_frame_refs,bin_", [(False, 1.0), (True, 1.0), (False, 2.0), (True, 2.0)])
def test_refs_two_spectrum_sets(gpu, two_frame_refs, bin_):
    rng = np.random.default_rng(7)
    nz, ny, nx = 3, 220, 212
    frames = rng.integers(0, 60, (nz, ny, nx)).astype(np.uint8)
    dark = rng.normal(1, 0.1, (ny, nx)).astype(np.float32)
    norm = rng.normal(1, 0.05, (ny, nx)).astype(np.float32)
    refs = {"dark": dark, "norm": norm}
    if two_frame_refs:
        refs["dark2"] = rng.normal(1, 0.1, (ny, nx)).astype(np.float32)
        refs["norm2"] = rng.normal(1, 0.05, (ny, nx)).astype(np.float32)
    p = api.verify_params(api.Params(bin=bin_, FrameDistOffset=0), nz)
    with api.Plan(p, nx, ny, nz, 0) as pl:
        pl.set_refs(**refs)
        pl.load_frames(frames)
        pl.forward()
        nu = O.verify_crop_size(nx, ny, 0, 0, 0, bin_)
        n = O.binned_size(nu, bin_)
        for f in range(nz):
            a, b = O.apply_refs(O.decode_frame(frames[f], 0), refs.get("dark"), refs.get("dark2"),
                                refs.get("norm"), refs.get("norm2"))
            assert rel_l2(pl.spectrum(f, 0), O.forward_spectrum(a, 0, 0, nu, n)) < SPEC_RTOL
            assert rel_l2(pl.spectrum(f, 1), O.forward_spectrum(b, 0, 0, nu, n)) < SPEC_RTOL


# ------------------------------------------------------------------ pairs --
@pytest.mark.parametrize("n,box,nps,fod", [(256, 96, 0, 2), (240, 64, 0, 3), (212, 95, 0, 2), (256, 48, 3, 2),
                                           (256, 16, 0, 2),
                                           # a large prime factor: generic column kernel, length-n outer table
                                           (514, 64, 0, 2), (502, 128, 0, 3)])
def test_pair_boxes_and_peaks(gpu, n, box, nps, fod):
    mv = synth.make_movie(n + 6, n + 2, 8, mean=1.5, seed=n + box, dtype="f32", speed=0.7, rw_sigma=0.4)
    params = api.Params(CCPeakSearchDim=box, NoisePeakSize=nps, FrameDistOffset=fod)
    p = api.verify_params(params, 8)
    with api.Plan(p, n + 6, n + 2, 8, 2) as pl:
        pl.load_frames(mv.frames)
        pl.forward()
        pl.pairs()
        gb = pl.boxes()
        gres = pl.pair_results()
    ob, _, _ = oracle_boxes(mv.frames, 2, p)
    for r in range(len(ob)):
        assert rel_l2(gb[r], ob[r]) < 1e-5
    ref = O.align_movie(mv.frames, 2, to_oparams(p))
    check_pairs(gres, ref, n, nps, ob)


# ---------------------------------------------------------- whole pipeline --
def compare_full(g, ref, n, nps, boxes=None):
    check_pairs(g, ref, n, nps, boxes)
    fo = np.stack([ref.frame_shift.real, ref.frame_shift.imag], 1)
    assert np.max(np.abs(g["frame_shifts"] - fo)) <= SHIFT_TOL
    assert rel_l2(g["image"], ref.image) <= IMAGE_RTOL


@pytest.mark.parametrize("n,box,nz", [(1024, 16, 8), (1024, 95, 8), (1024, 256, 6), (2048, 128, 6), (4096, 96, 5)])
def test_pair_boxes_compiled_splits(gpu, n, box, nz):
    """The pair kernels with the split n = P*Q compiled in (1024 = 32*32,
    2048 = 32*64, 4096 = 64*64 under the tuned schedules): column-stage Horner
    sums and the pruned-transform row stage at box sizes other than 96, odd
    included, against the oracle's windows and peaks."""
    mv = synth.make_movie(n + 4, n, nz, mean=1.0, seed=n + box, dtype="u8", speed=0.7, rw_sigma=0.4)
    p = api.verify_params(api.Params(CCPeakSearchDim=box, FrameDistOffset=1), nz)
    with api.Plan(p, n + 4, n, nz, 0) as pl:
        assert pl.info["prune_p"] * pl.info["prune_q"] == n and pl.info["prune_p"] <= 128
        pl.load_frames(mv.frames)
        pl.forward()
        pl.pairs()
        gb = pl.boxes()
        gres = pl.pair_results()
    ob, _, _ = oracle_boxes(mv.frames, 0, p)
    for r in range(len(ob)):
        assert rel_l2(gb[r], ob[r]) < 1e-5, r
    ref = O.align_movie(mv.frames, 0, to_oparams(p))
    check_pairs(gres, ref, n, p.NoisePeakSize, ob)


def test_pipeline_c1_shape(gpu):
    """c1 geometry: 16 x 1024^2 float32, -fod 2 -bft 150 -pbx 96."""
    mv = synth.make_movie(1024, 1024, 16, mean=1.5, seed=11, dtype="f32", speed=0.4, rw_sigma=0.3)
    g, ref, p = run_both(mv.frames, 2, api.Params(FrameDistOffset=2))
    compare_full(g, ref, 1024, 0)
    truth_rmse = np.sqrt(np.mean(np.sum((g["frame_shifts"] + (mv.truth - mv.truth[0])) ** 2, 1)))
    assert truth_rmse < 0.2


@pytest.mark.parametrize("seed,kw", [
    (1, dict(bAlignToMid=0)),
    (2, dict(nStart=2, nEnd=9, nStartSum=3, nEndSum=8)),
    (3, dict(iter=3, iterthres=0.001)),
    (4, dict(kiThresh=0.05)),
    (5, dict(bfactor=40.0, CCPeakSearchDim=64)),
])
def test_pipeline_options(gpu, seed, kw):
    mv = synth.make_movie(300, 290, 12, mean=2.0, seed=seed, dtype="u8", speed=0.6, rw_sigma=0.4)
    g, ref, p = run_both(mv.frames, 0, api.Params(**kw))
    compare_full(g, ref, ref.nsam, p.NoisePeakSize)


def test_pipeline_bin2_radix53(gpu):
    """-bin 2 from 424 to 212 = 4*53: radix-53 butterflies in both passes."""
    mv = synth.make_movie(430, 424, 8, mean=0.5, seed=5, dtype="u8", speed=1.0, rw_sigma=0.5)
    g, ref, p = run_both(mv.frames, 0, api.Params(bin=2.0, CCPeakSearchDim=64))
    compare_full(g, ref, 212, 0)


def test_pipeline_refs(gpu):
    mv = synth.make_movie(256, 256, 8, mean=3.0, seed=9, dtype="u8", speed=0.8, rw_sigma=0.3)
    rng = np.random.default_rng(1)
    refs = {"dark": rng.normal(0.2, 0.02, (256, 256)).astype(np.float32),
            "norm": rng.normal(1.0, 0.02, (256, 256)).astype(np.float32)}
    g, ref, p = run_both(mv.frames, 0, api.Params(), refs=refs)
    compare_full(g, ref, 256, 0)


@pytest.mark.parametrize("stretch,refs,kw", [
    ((1.03, 1.0), None, dict()),
    ((1.0, 1.05), "one", dict(crop_offsetx=3, crop_offsety=2)),
    ((1.02, 1.04), "two", dict(bin=2.0, CCPeakSearchDim=64)),
])
def test_pipeline_stretch(gpu, stretch, refs, kw):
    """-scx/-scy: the nearest-neighbour stretch after dark/gain
    (DFAlign.cu:751-765), with one- and two-frame references."""
    mv = synth.make_movie(300, 290, 8, mean=2.0, seed=21, dtype="u8", speed=0.6, rw_sigma=0.4)
    rng = np.random.default_rng(22)
    r = None
    if refs:
        r = {"dark": rng.normal(0.2, 0.05, (290, 300)).astype(np.float32),
             "norm": rng.normal(1.0, 0.05, (290, 300)).astype(np.float32)}
        if refs == "two":
            r["dark2"] = rng.normal(0.3, 0.05, (290, 300)).astype(np.float32)
            r["norm2"] = rng.normal(1.0, 0.05, (290, 300)).astype(np.float32)
    g, ref, p = run_both(mv.frames, 0, api.Params(**kw), refs=r, stretch=stretch)
    compare_full(g, ref, ref.nsam, p.NoisePeakSize)
    plain = O.align_movie(mv.frames, 0, to_oparams(p), refs=r)
    assert rel_l2(plain.image, ref.image) > 1e-3  # the stretch changed the input


def test_stretch_switch_and_limits(gpu):
    """Stretch on, off again and refs set after it: every run matches the
    oracle (no captured movie keeps stale pointers); factors < 1 refused."""
    mv = synth.make_movie(256, 256, 6, mean=2.0, seed=23, dtype="u8", speed=0.6, rw_sigma=0.4)
    p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=1), 6)
    rng = np.random.default_rng(24)
    refs = {"dark": rng.normal(0.2, 0.05, (256, 256)).astype(np.float32)}
    with api.Plan(p, 256, 256, 6, 0) as pl:
        pl.load_frames(mv.frames)
        for st, rf in [((1.0, 1.0), None), ((1.04, 1.0), None), ((1.04, 1.0), refs), ((1.0, 1.0), refs)]:
            pl.set_stretch(*st)
            if rf is not None:
                pl.set_refs(**rf)
            img = pl.run()
            want = O.align_movie(mv.frames, 0, to_oparams(p), refs=rf, stretch=st).image
            assert rel_l2(img, want) <= IMAGE_RTOL
        with pytest.raises(Exception, match="X-axis"):
            pl.set_stretch(0.9, 1.0)


@pytest.mark.slow
def test_pipeline_3710_crop(gpu):
    """The c2 crop side 3710 = 2*5*7*53 on a short stack (oracle cost bound)."""
    mv = synth.make_movie(3730, 3710, 6, mean=1.2, seed=2, dtype="u8", speed=0.3, rw_sigma=0.5)
    g, ref, p = run_both(mv.frames, 0, api.Params(FrameDistOffset=1))
    assert ref.nsam == 3710
    compare_full(g, ref, 3710, 0)


@pytest.mark.slow
def test_pipeline_c3_geometry(gpu):
    """The c3 geometry (7676x7420 class, -bin 2: forward at 7420 = 2*3710,
    Fourier crop to 3710) on a short stack."""
    mv = synth.make_movie(7440, 7420, 4, mean=0.3, seed=12, dtype="u8", speed=0.3, rw_sigma=0.5)
    g, ref, p = run_both(mv.frames, 0, api.Params(bin=2.0, FrameDistOffset=1))
    assert (ref.nsam_unbin, ref.nsam) == (7420, 3710)
    compare_full(g, ref, 3710, 0)


@pytest.mark.parametrize("n,q,ppc", [(256, 8, 4), (240, 16, 3), (256, 64, 64), (256, 32, 7)])
def test_pair_boxes_scheduled(gpu, n, q, ppc):
    """Schedules other than the built-in choice (split n = P*Q, pairs per CTA,
    a last CTA with fewer pairs) against the oracle's CC windows."""
    mv = synth.make_movie(n + 6, n, 8, mean=1.5, seed=n + q, dtype="f32", speed=0.7, rw_sigma=0.4)
    p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=2), 8)
    api.schedule_set(n, pair_q=q, pairs_per_cta=ppc)
    try:
        with api.Plan(p, n + 6, n, 8, 2) as pl:
            assert (pl.info["prune_p"], pl.info["prune_q"]) == (n // q, q)
            pl.load_frames(mv.frames)
            pl.forward()
            pl.pairs()
            gb = pl.boxes()
            gres = pl.pair_results()
    finally:
        api.schedule_clear()
    ob, _, _ = oracle_boxes(mv.frames, 2, p)
    for r in range(len(ob)):
        assert rel_l2(gb[r], ob[r]) < 1e-5
    ref = O.align_movie(mv.frames, 2, to_oparams(p))
    check_pairs(gres, ref, n, 0, ob)
