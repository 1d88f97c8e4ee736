"""The reference's whole program against the oracle and this path, on the GPU.

oracle/_ref/dosefgpu_driftcorr_ref is the reference's own dosefgpu_driftcorr
built from its sources by oracle/build_ref.sh (DFAlign.cu, cufunc.cu with
cuFFT, func.cpp, the MRC readers) with three project stand-ins for libraries
that are not installed: SP++ (oracle/stubs/sppp: Matrix/Vector, Householder
least squares, one-sided Jacobi SVD rank), FFTW (cuFFT's FFTW interface) and
libtiff (TIFF input refused).  Every run uses -dsp 0.

What these tests pin:
  * the pair stage: the reference's pair shifts against the FP64 oracle's
    (equal on the 1/32 grid except documented near-ties);
  * the drift solve: the reference's own lsSolver + OD_Threshold
    (DFAlign.cu:914-948, mfunc.h:101-146) -- its ki lines, kept pairs and
    frame shifts against the oracle's solve of the reference's own pair
    shifts;
  * the realignment iterations (DFAlign.cu:950-1071): the reference's
    per-iteration frame-vs-sum shifts and final shifts against this path's
    CLI and the oracle;
  * the sum (-fcs) against the oracle and this path.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from motioncorr1exp_b200 import mrc, synth
from oracle import mc_oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "dosefgpu_driftcorr_ref")
CLI = os.path.join(ROOT, "motioncorr1exp_b200", "lib", "dosefgpu_driftcorr")

PAIR_RE = re.compile(r"\.\.\.\.\.\.(\d+) Frame #(\d+) VS #(\d+) xy-shift:\s+(\S+)\s+(\S+)\s+CC:(\S+)")
KI_RE = re.compile(r"\.\.\.\.\.\.ki #(\d+) of Frame #(\d+) VS #(\d+):\s+(\S+)")
SHIFT_RE = re.compile(r"\.\.\.\.\.\.Shift of Frame #(\d+) : \s*(\S+)\s+(\S+)")
ITER_RE = re.compile(r"\.\.\.\.\.\.(\d+) Frame #(\d+) VS <sum> xy-shift:\s+(\S+)\s+(\S+) \(")


def parse_log(text):
    """Pair lines, both ki rounds, per-iteration frame-vs-sum lines and the
    final shifts of a DFAlign-format log."""
    out = {"pairs": [], "ki1": [], "ki2": [], "iter": [], "shift": []}
    rnd = None
    for line in text.splitlines():
        if "ki: First round" in line:
            rnd = "ki1"
        elif "ki: Second round" in line:
            rnd = "ki2"
        elif line.startswith("Iteration ["):
            out["iter"].append([])
        m = PAIR_RE.search(line)
        if m:
            out["pairs"].append((int(m[2]), int(m[3]), float(m[4]), float(m[5]), float(m[6])))
            continue
        m = KI_RE.search(line)
        if m and rnd:
            out[rnd].append((int(m[2]), int(m[3]), float(m[4])))
            continue
        m = ITER_RE.search(line)
        if m:
            out["iter"][-1].append((float(m[3]), float(m[4])))
            continue
        m = SHIFT_RE.search(line)
        if m:
            out["shift"].append((float(m[2]), float(m[3])))
    return out


def on_grid(v):
    """A printed (%8.4f) pair shift back on its exact 1/32-px grid point."""
    return np.round(np.asarray(v, dtype=np.float64) * 32.0) / 32.0


def run_prog(exe, stack, outdir, flags, tag):
    log = os.path.join(outdir, f"{tag}_log.txt")
    fcs = os.path.join(outdir, f"{tag}_sum.mrc")
    args = [exe, stack, "-dsp", "0", "-fcs", fcs, "-flg", log] + [str(f) for f in flags]
    r = subprocess.run(args, cwd=outdir, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"{tag}: rc {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}"
    text = open(log).read() if os.path.exists(log) else r.stdout
    return parse_log(text), mrc.read_stack(fcs)[0][0].astype(np.float64)


@pytest.fixture(scope="module")
def ref_exe():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/dosefgpu_driftcorr_ref not built (reference tree absent where built)")
    return REF


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_params(flags, nz):
    kv = dict(zip(flags[::2], flags[1::2]))
    p = O.Params(FrameDistOffset=int(kv.get("-fod", 2)), bfactor=float(kv.get("-bft", 150)),
                 CCPeakSearchDim=int(kv.get("-pbx", 96)), NoisePeakSize=int(kv.get("-nps", 0)),
                 kiThresh=float(kv.get("-kit", 1.0)), bAlignToMid=int(kv.get("-atm", 1)),
                 iter=int(kv.get("-itr", 0)), iterthres=float(kv.get("-ith", 0.0)), bin=float(kv.get("-bin", 1.0)))
    return O.verify_para(p, nz)


def solve_from_pairs(pairs, nframe, kithresh):
    """The oracle's FP64 solve (DFAlign.cu:914-948) of printed pair shifts."""
    ij = [(i, j) for i, j, *_ in pairs]
    b = np.array([complex(sx, sy) for sx, sy in on_grid([(p[2], p[3]) for p in pairs])])
    A = O.design_matrix(ij, nframe)
    s = O.lsq(A, b)
    ki1 = np.abs(A @ s - b)
    good = O.od_threshold(A, b, ki1, kithresh)
    s2 = O.lsq(A[good], b[good])
    ki2 = np.abs(A[good] @ s2 - b[good])
    return ij, ki1, good, ki2, np.concatenate([[0], np.cumsum(s2)])


CASES = {
    # c1's shape: 16 x 1024^2 float32, -fod 2 -nps 0
    "c1": dict(nx=1024, ny=1024, nz=16, mean=1.5, dtype="f32", speed=0.4, rw=0.3, seed=11,
               flags=["-fod", "2", "-bft", "150", "-pbx", "96", "-nps", "0"]),
    # c1 with three realignment iterations
    "c1_itr3": dict(nx=1024, ny=1024, nz=16, mean=1.5, dtype="f32", speed=0.4, rw=0.3, seed=12,
                    flags=["-fod", "2", "-itr", "3", "-ith", "0.0"]),
    # the c2 frame size (crop 3710: radix 53), 12 frames, noisier drift, -kit 0.3
    "c2_12": dict(nx=3838, ny=3710, nz=12, mean=1.2, dtype="u8", speed=0.3, rw=0.5, seed=13,
                  flags=["-fod", "2", "-atm", "1", "-kit", "0.3"]),
    # super-resolution frames binned by 2 in Fourier space (7420 -> 3710), 6 frames
    "c3_6": dict(nx=7676, ny=7420, nz=6, mean=0.3, dtype="u8", speed=0.3, rw=0.5, seed=14,
                 flags=["-bin", "2", "-fod", "1", "-itr", "2"]),
}


@pytest.mark.parametrize("name", list(CASES))
def test_reference_program(gpu, ref_exe, tmp_path, name):
    c = CASES[name]
    mv = synth.make_movie(c["nx"], c["ny"], c["nz"], mean=c["mean"], seed=c["seed"], dtype=c["dtype"],
                          speed=c["speed"], rw_sigma=c["rw"])
    stack = str(tmp_path / "movie.mrc")
    mrc.write_stack(stack, mv.frames, mv.mode)
    ref, ref_img = run_prog(ref_exe, stack, str(tmp_path), c["flags"], "ref")
    ours, our_img = run_prog(CLI, stack, str(tmp_path), c["flags"], "ours")
    p = oracle_params(c["flags"], c["nz"])
    orc = O.align_movie(mv.frames, mv.mode, p)
    nframe = len(orc.frame_shift)
    P = len(orc.pairs)

    # pair stage: the reference's FP32 cuFFT shifts vs the FP64 oracle
    assert [(i, j) for i, j, *_ in ref["pairs"]] == [tuple(q) for q in orc.pairs]
    rs = on_grid([(q[2], q[3]) for q in ref["pairs"]])
    os_ = np.stack([orc.pair_shift.real, orc.pair_shift.imag], 1)
    flips = int(np.sum(np.any(rs != os_, axis=1)))
    assert flips <= max(1, P // 50), f"{flips} of {P} reference pair shifts off the oracle's grid point"
    assert np.max(np.abs(rs - os_)) <= 2.0 / 32 + 1e-9

    # drift solve: the reference's own lsSolver / OD_Threshold on its own pair
    # shifts against the oracle's solve of the same shifts
    ij, ki1, good, ki2, fs = solve_from_pairs(ref["pairs"], nframe, float(p.kiThresh))
    np.testing.assert_allclose([k[2] for k in ref["ki1"]], ki1, atol=0.6e-4)
    assert [(k[0], k[1]) for k in ref["ki2"]] == [ij[g] for g in good]
    np.testing.assert_allclose([k[2] for k in ref["ki2"]], ki2, atol=0.6e-4)
    if p.iter == 0:
        np.testing.assert_allclose(np.array(ref["shift"]), np.stack([fs.real, fs.imag], 1), atol=0.6e-4)

    # this path's CLI prints the reference's lines; where both pair stages
    # land on the same grid points everything downstream agrees to print
    # precision
    gs = on_grid([(q[2], q[3]) for q in ours["pairs"]])
    same_pairs = bool(np.array_equal(gs, rs))
    if same_pairs:
        assert [(k[0], k[1]) for k in ours["ki2"]] == [(k[0], k[1]) for k in ref["ki2"]]
        np.testing.assert_allclose([k[2] for k in ours["ki1"]], [k[2] for k in ref["ki1"]], atol=1.1e-4)
        if p.iter == 0:
            np.testing.assert_allclose(np.array(ours["shift"]), np.array(ref["shift"]), atol=1.1e-4)

    # realignment iterations: frame-vs-sum shifts of every iteration
    assert len(ref["iter"]) == len(orc.iter_log) == len(ours["iter"])
    for it, (r_it, o_it) in enumerate(zip(ref["iter"], orc.iter_log)):
        r_arr = on_grid(r_it)
        o_arr = np.stack([o_it["newshift"].real, o_it["newshift"].imag], 1)
        if same_pairs and it == 0:
            assert int(np.sum(np.any(r_arr != o_arr, axis=1))) <= max(1, nframe // 8)
    # final shifts: reference vs oracle and ours vs reference within 0.01 px
    fo = np.stack([orc.frame_shift.real, orc.frame_shift.imag], 1)
    assert np.max(np.abs(np.array(ref["shift"]) - fo)) <= 0.01 + 0.6e-4 or flips > 0
    assert np.max(np.abs(np.array(ours["shift"]) - np.array(ref["shift"]))) <= 0.01 + 1.1e-4 or not same_pairs

    # sums: both within 1e-5 of the oracle (relative L2) where the shifts agree
    if same_pairs and flips == 0:
        assert rel_l2(ref_img, orc.image) <= 1e-5
        assert rel_l2(our_img, orc.image) <= 1e-5
        assert rel_l2(our_img, ref_img) <= 2e-5
    print(f"{name}: {P} pairs, reference-vs-oracle grid flips {flips}, same pairs as ours {same_pairs}, "
          f"sum rel L2 ref {rel_l2(ref_img, orc.image):.2e} ours {rel_l2(our_img, orc.image):.2e}")
