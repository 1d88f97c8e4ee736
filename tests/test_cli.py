"""dosefgpu_driftcorr CLI: flags, defaults, aborts and the parameter log of
dosefgpu_driftcorr.cpp (CPU: every case here stops before the GPU), and a
full run on a small stack (GPU)."""
import os
import re
import subprocess

import numpy as np
import pytest

from motioncorr1exp_b200 import api, mrc, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "motioncorr1exp_b200", "lib", "dosefgpu_driftcorr")


def run(args, cwd):
    r = subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout + r.stderr


@pytest.fixture
def stack(tmp_path):
    frames = np.random.default_rng(0).integers(0, 5, (6, 40, 48)).astype(np.uint8)
    p = tmp_path / "movie.mrc"
    mrc.write_stack(str(p), frames, 0)
    return p


def test_usage_without_arguments(tmp_path):
    rc, out = run([], tmp_path)
    assert rc == 0
    assert "-fod       2" in out and "-bft       150" in out and "-pbx       96" in out


@pytest.mark.parametrize("args,msg", [
    (["-fod"], "Wrong number of arguments. Abort."),
    (["-xyz", "1"], "Undefined option: -xyz .Abort."),
    (["-fod", "3"], "Frame distance offset is too big or less than 0. Abort"),
    (["-fod", "-1"], "Frame distance offset is too big or less than 0. Abort"),
    (["-scx", "0.5"], "Stretching factor along X-axis needs to be >=1.0."),
    (["-scy", "0.9"], "Stretching factor along Y-axis needs to be >=1.0."),
    (["-2es", "5", "-nes", "4"], "Last frame # for the second sum image cannot be larger"),
])
def test_abort_messages(stack, args, msg):
    rc, out = run([str(stack)] + args, stack.parent)
    assert rc == 1
    assert msg in out
    assert "Error: Have wrong parameters. Abort!" in out


def test_bin_clamp_messages(stack):
    rc, out = run([str(stack), "-bin", "3", "-fod", "9"], stack.parent)
    assert "Larger than maximum binning 2. Set to 2." in out
    rc, out = run([str(stack), "-bin", "0.5", "-fod", "9"], stack.parent)
    assert "Smaller than minimum binning 1. Set to 1." in out


def test_not_a_stack(tmp_path):
    p = tmp_path / "one.mrc"
    mrc.write_stack(str(p), np.zeros((1, 8, 8), np.uint8), 0)
    rc, out = run([str(p)], tmp_path)
    assert rc == 1 and "Not a stack or wrong file. Abort" in out


def test_parameter_log_and_default_names(stack, tmp_path):
    # valid parameters: ShowPara writes the log before the alignment starts
    subprocess.run([CLI, str(stack), "-fod", "1", "-bft", "120", "-nst", "1", "-dsp", "0"], cwd=tmp_path,
                   capture_output=True, text=True, timeout=300)
    log = (tmp_path / "movie_Log.txt").read_text()
    assert log.startswith("******Parameter List******\n")
    assert f"Input:  {stack}\n" in log
    assert "  -bft  120.000000\n" in log
    assert "  -fod  1\n" in log
    assert "  -nst  1\n" in log
    assert "  -ned  5\n" in log           # repaired by VerifyPara
    assert "  -fcs  movie_SumCorr.mrc\n" in log
    assert "  -dsp  0\n" in log
    assert "******Parameter End******\n" in log


@pytest.mark.gpu
def test_cli_full_run_matches_api(gpu, tmp_path):
    mv = synth.make_movie(200, 190, 8, mean=2.0, seed=4, dtype="u8", speed=0.8, rw_sigma=0.3)
    p = tmp_path / "m.mrc"
    mrc.write_stack(str(p), mv.frames, 0)
    rc, out = run([str(p), "-pbx", "64", "-fod", "2", "-dsp", "0", "-fcs", "sum.mrc", "-flg", "log.txt"], tmp_path)
    assert rc == 0, out
    img = mrc.read_image(str(tmp_path / "sum.mrc"))
    res = api.align(mv.frames, 0, api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=2), 8))
    np.testing.assert_allclose(img, res["image"], rtol=0, atol=1e-5 * np.abs(res["image"]).max())
    log = (tmp_path / "log.txt").read_text()
    got = [(float(a), float(b)) for a, b in re.findall(r"Shift of Frame #\d{3} : +(\S+) +(\S+)", log)]
    np.testing.assert_allclose(np.array(got), np.round(res["frame_shifts"], 4), atol=1.1e-4)
    assert "Save Sum to: sum.mrc" in log and "Done." in log
    h = mrc.read_header(str(tmp_path / "sum.mrc"))
    assert int(h["mode"]) == 2 and bytes(h["map"]) == b""


@pytest.mark.gpu
def test_cli_extra_outputs(gpu, tmp_path):
    """-srs (unaligned sum), -2es (second sum), -ssc (aligned stack) and -sub
    names, with their log lines where the reference prints them."""
    mv = synth.make_movie(200, 190, 10, mean=2.0, seed=5, dtype="u8", speed=0.8, rw_sigma=0.3)
    p = tmp_path / "m.mrc"
    mrc.write_stack(str(p), mv.frames, 0)
    rc, out = run([str(p), "-pbx", "64", "-fod", "2", "-dsp", "0", "-srs", "1", "-ssc", "1", "-2es", "5",
                   "-nss", "1", "-flg", "log.txt"], tmp_path)
    assert rc == 0, out
    prm = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=2, nStartSum=1), 10)
    with api.Plan(prm, 200, 190, 10, 0) as pl:
        pl.load_frames(mv.frames)
        img = pl.run()
        raw, sum2 = pl.raw_sum(), pl.sum_to(5)
        stack = np.stack([pl.corrected_frame(k) for k in range(1, 10)])
    tol = 1e-5 * np.abs(img).max()
    np.testing.assert_allclose(mrc.read_image(str(tmp_path / "m_SumCorr.mrc")), img, rtol=0, atol=tol)
    np.testing.assert_allclose(mrc.read_image(str(tmp_path / "m_SumRaw.mrc")), raw, rtol=0, atol=tol)
    np.testing.assert_allclose(mrc.read_image(str(tmp_path / "m_SumCorr2.mrc")), sum2, rtol=0, atol=tol)
    h = mrc.read_header(str(tmp_path / "m_Corrected.mrc"))
    assert (int(h["nx"]), int(h["ny"]), int(h["nz"]), int(h["mode"])) == (190, 190, 9, 2)
    got = np.fromfile(str(tmp_path / "m_Corrected.mrc"), dtype=np.float32, offset=1024).reshape(9, 190, 190)
    np.testing.assert_allclose(got, stack, rtol=0, atol=tol)
    log = (tmp_path / "log.txt").read_text()
    lines = log.splitlines()
    i_raw = lines.index("Save Unaligned Sum to: m_SumRaw.mrc")
    i_pair = lines.index("Calculate relative drift between frames")
    i_read = max(i for i, l in enumerate(lines) if l.startswith("......Read and sum frame"))
    assert i_read < i_raw < i_pair
    i_add5 = next(i for i, l in enumerate(lines) if l.startswith("......Add Frame #005"))
    assert lines[i_add5 + 2] == "Save Sum to: m_SumCorr2.mrc"
    assert lines[i_add5 + 3].startswith("......Add Frame #006")
    # -sub: crop-tagged names of both sums
    rc, out = run([str(p), "-pbx", "64", "-fod", "2", "-dsp", "0", "-sub", "1", "-2es", "5", "-crx", "4"],
                  tmp_path)
    assert rc == 0, out
    assert (tmp_path / "m_SumCorr_ox4_oy0_dim190.mrc").exists()
    assert (tmp_path / "m_SumCorr2_ox4_oy0_dim190.mrc").exists()


@pytest.mark.gpu
def test_cli_quicklook_displays(gpu, tmp_path):
    """-dsp 1 (the default): three 400 x 400 mode-1 displays in ./dosef_quick,
    equal to the C ABI's; below 400 pixels the run warns and still saves."""
    mv = synth.make_movie(520, 512, 6, mean=2.0, seed=6, dtype="u8", speed=0.6, rw_sigma=0.3)
    p = tmp_path / "m.mrc"
    mrc.write_stack(str(p), mv.frames, 0)
    rc, out = run([str(p), "-pbx", "64", "-fod", "1"], tmp_path)
    assert rc == 0, out
    prm = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=1), 6)
    with api.Plan(prm, 520, 512, 6, 0) as pl:
        pl.load_frames(mv.frames)
        pl.run()
        want = {k: pl.quicklook(v) for k, v in (("RawFFT", "raw_fft"), ("CorrSum", "corr_sum"),
                                                  ("CorrFFT", "corr_fft"))}
    for k, w in want.items():
        f = tmp_path / "dosef_quick" / f"m_{k}.mrc"
        h = mrc.read_header(str(f))
        assert (int(h["nx"]), int(h["ny"]), int(h["nz"]), int(h["mode"])) == (400, 400, 1, 1)
        got = np.fromfile(str(f), dtype=np.int16, offset=1024).reshape(400, 400)
        np.testing.assert_array_equal(got, w)
        assert float(h["dmin"]) == w.min() and float(h["dmax"]) == w.max()
    small = tmp_path / "s.mrc"
    mrc.write_stack(str(small), mv.frames[:, :200, :200].copy(), 0)
    rc, out = run([str(small), "-pbx", "64", "-fod", "1", "-flg", "s.txt"], tmp_path)
    assert rc == 0, out
    assert "Warning: display ./dosef_quick/s_RawFFT.mrc not written" in (tmp_path / "s.txt").read_text()
    assert (tmp_path / "s_SumCorr.mrc").exists()


def _tiff(path, frames, **kw):
    from PIL import Image
    ims = [Image.fromarray(f) for f in frames]
    ims[0].save(str(path), save_all=True, append_images=ims[1:], **kw)


def test_tiff_and_mrcgz_stacks_pass_verify(tmp_path):
    """TIFF and MRC-gz stacks are detected and counted (getNFrame,
    DFAlign.cu:344-368): a bad -fod then aborts as for MRC."""
    pytest.importorskip("PIL")
    import gzip
    frames = np.random.default_rng(1).integers(0, 5, (6, 40, 48)).astype(np.uint8)
    _tiff(tmp_path / "m.tif", frames, compression="tiff_lzw")
    mrc.write_stack(str(tmp_path / "m.mrc"), frames, 0)
    (tmp_path / "m.mrc.gz").write_bytes(gzip.compress((tmp_path / "m.mrc").read_bytes()))
    for name in ("m.tif", "m.mrc.gz"):
        rc, out = run([str(tmp_path / name), "-fod", "9"], tmp_path)
        assert rc == 1 and "Frame distance offset is too big" in out and "Not a stack" not in out
    (tmp_path / "x.txt").write_text("hello" * 300)
    rc, out = run([str(tmp_path / "x.txt")], tmp_path)
    assert rc == 1 and "Not a stack or wrong file. Abort" in out


@pytest.mark.gpu
def test_cli_tiff_and_mrcgz_runs(gpu, tmp_path):
    """One movie as MRC, 8-bit LZW TIFF, 16-bit Deflate TIFF and MRC-gz: the
    same aligned sum; the TIFF log names mode 7199 as the reference does."""
    pytest.importorskip("PIL")
    import gzip
    mv = synth.make_movie(200, 190, 8, mean=2.0, seed=7, dtype="u8", speed=0.8, rw_sigma=0.3)
    mrc.write_stack(str(tmp_path / "a.mrc"), mv.frames, 0)
    _tiff(tmp_path / "b.tif", mv.frames, compression="tiff_lzw")
    _tiff(tmp_path / "c.tif", mv.frames.astype(np.uint16), compression="tiff_adobe_deflate")
    (tmp_path / "d.mrc.gz").write_bytes(gzip.compress((tmp_path / "a.mrc").read_bytes()))
    sums = {}
    for name in ("a.mrc", "b.tif", "c.tif", "d.mrc.gz"):
        stem = name[0]
        rc, out = run([str(tmp_path / name), "-pbx", "64", "-fod", "2", "-dsp", "0", "-flg", stem + ".txt"],
                      tmp_path)
        assert rc == 0, out
        # default names drop only the last extension (dosefgpu_driftcorr.cpp:433-481)
        sums[stem] = mrc.read_image(str(tmp_path / f"{name[:name.rfind('.')]}_SumCorr.mrc"))
        log = (tmp_path / f"{stem}.txt").read_text()
        mode = 7199 if name.endswith(".tif") else 0
        assert f"Input Stack: Nx(200) Ny(190) Nz(8) Mode({mode})" in log
        fmt = {"a": "MRC2000", "b": "TIFF", "c": "TIFF", "d": "MRC-gz"}[stem]
        assert f"Auto-detected file format: {fmt}" in out
    for k in ("b", "c", "d"):
        np.testing.assert_array_equal(sums[k], sums["a"])


@pytest.mark.gpu
def test_cli_fsc_and_ccmap(gpu, tmp_path):
    """-fsc 1: PlotFSC's table after the sum (DFAlign.cu:309-319); -scc 1: the
    pair CC windows as a box x box x npairs float stack, logged after the
    final shifts (DFAlign.cu:1094-1099)."""
    mv = synth.make_movie(520, 512, 8, mean=2.0, seed=8, dtype="u8", speed=0.8, rw_sigma=0.3)
    p = tmp_path / "m.mrc"
    mrc.write_stack(str(p), mv.frames, 0)
    rc, out = run([str(p), "-pbx", "64", "-fod", "2", "-dsp", "0", "-fsc", "1", "-scc", "1", "-flg", "log.txt"],
                  tmp_path)
    assert rc == 0, out
    prm = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=2), 8)
    with api.Plan(prm, 520, 512, 8, 0) as pl:
        pl.load_frames(mv.frames)
        pl.run()
        fsc = pl.fsc()
        boxes = pl.boxes()
        npairs = pl.npairs
    lines = (tmp_path / "log.txt").read_text().splitlines()
    i = lines.index("FSC parallel(D) and perpendicular(U) to drift direction:")
    assert lines[i - 2].startswith("Save Sum to: m_SumCorr.mrc") and lines[i - 1] == ""
    assert lines[i + 1] == "   Nq%       D_Raw       U_Raw       D_Corr       U_Corr"
    rows = lines[i + 2:i + 2 + len(fsc)]
    want = ["%7.2f %12.4f %12.4f %12.4f %12.4f" % tuple(r) for r in fsc]
    assert rows == want
    assert lines[i + 2 + len(fsc)] == "" and lines[-1] == "Done."
    h = mrc.read_header(str(tmp_path / "m_CCMap.mrc"))
    assert (int(h["nx"]), int(h["ny"]), int(h["nz"]), int(h["mode"])) == (64, 64, npairs, 2)
    got = np.fromfile(str(tmp_path / "m_CCMap.mrc"), dtype=np.float32, offset=1024).reshape(boxes.shape)
    np.testing.assert_array_equal(got, boxes)
    j = lines.index("Save CC map to: m_CCMap.mrc")
    assert lines[j - 1].startswith("......Shift of Frame #007")


@pytest.mark.gpu
def test_cli_stretch(gpu, tmp_path):
    """-scx/-scy reach the plan: the CLI's sum equals the API's with the same
    stretch and differs from the unstretched one."""
    mv = synth.make_movie(200, 190, 8, mean=2.0, seed=9, dtype="u8", speed=0.8, rw_sigma=0.3)
    p = tmp_path / "m.mrc"
    mrc.write_stack(str(p), mv.frames, 0)
    rc, out = run([str(p), "-pbx", "64", "-fod", "2", "-dsp", "0", "-scx", "1.04", "-scy", "1.02"], tmp_path)
    assert rc == 0, out
    img = mrc.read_image(str(tmp_path / "m_SumCorr.mrc"))
    prm = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=2), 8)
    want = api.align(mv.frames, 0, prm, stretch=(1.04, 1.02))["image"]
    np.testing.assert_array_equal(img, want)
    assert not np.array_equal(img, api.align(mv.frames, 0, prm)["image"])
