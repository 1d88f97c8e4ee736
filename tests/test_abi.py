"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and its host-only entry points (defaults, VerifyPara, the
FP64 drift solve) agree with the reference semantics / the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from motioncorr1exp_b200 import _lib, api
from oracle import mc_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "mc.h")).read()
    return sorted(set(re.findall(r"\b(mc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
        assert s in _lib.SIGNATURES, f"{s} declared in mc.h but not bound"


def test_version_and_errors():
    L = _lib.lib()
    assert L.mc_version() == 10000
    assert L.mc_strerror(0) == b"ok"
    assert L.mc_strerror(-4) == b"unsupported size"


def test_default_params_match_getDefaultPara():
    p = api.default_params()
    o = O.Params()
    for k in ("crop_offsetx", "crop_offsety", "crop_nsam", "bin", "bfactor", "CCPeakSearchDim",
              "FrameDistOffset", "NoisePeakSize", "kiThresh", "bAlignToMid", "iter", "iterthres"):
        assert getattr(p, k) == getattr(o, k), k


def test_verify_params_repairs_and_aborts():
    p = api.verify_params(api.Params(nStart=-3, nEnd=0, nStartSum=0, nEndSum=0), 20)
    assert (p.nStart, p.nEnd, p.nStartSum, p.nEndSum) == (0, 19, 0, 19)
    p = api.verify_params(api.Params(nStart=5, nEnd=50, nStartSum=2, nEndSum=8), 20)
    assert (p.nStart, p.nEnd, p.nStartSum, p.nEndSum) == (5, 19, 5, 8)
    with pytest.raises(_lib.McError) as e:
        api.verify_params(api.Params(FrameDistOffset=10), 20)
    assert "Frame distance offset is too big" in str(e.value)
    with pytest.raises(_lib.McError):
        api.verify_params(api.Params(), 1)


def test_plan_create_rejects_bad_geometry_without_gpu():
    # argument checks run before any device call
    with pytest.raises(_lib.McError) as e:
        api.Plan(api.Params(), 100, 100, 10, mode=5)
    assert e.value.code == -1


@pytest.mark.parametrize("nframe,fod,seed", [(10, 2, 0), (16, 2, 1), (24, 5, 2)])
def test_solve_pairs_matches_oracle(nframe, fod, seed):
    rng = np.random.default_rng(seed)
    pairs = O.pair_list(nframe, fod)
    A = O.design_matrix(pairs, nframe)
    steps = rng.normal(0, 1, nframe - 1) + 1j * rng.normal(0, 1, nframe - 1)
    b = A @ steps + (rng.normal(0, 0.05, len(pairs)) + 1j * rng.normal(0, 0.05, len(pairs)))
    b[3] += 4.0 - 2.0j   # an outlier
    b = np.round(b * 32) / 32          # pair shifts are 1/32-px quantised floats
    shifts = np.stack([b.real, b.imag], 1).astype(np.float32)
    got = api.solve_pairs(nframe, np.array(pairs), shifts, 1.0)
    bo = shifts[:, 0].astype(np.float64) + 1j * shifts[:, 1]
    s1 = O.lsq(A, bo)
    ki1 = np.abs(A @ s1 - bo)
    np.testing.assert_allclose(got["ki1"], ki1, atol=1e-9)
    good = O.od_threshold(A, bo, ki1, 1.0)
    assert list(got["kept"]) == good
    s2 = O.lsq(A[good], bo[good])
    np.testing.assert_allclose(got["step"][:, 0] + 1j * got["step"][:, 1], s2, atol=1e-9)
    np.testing.assert_allclose(got["ki2"], np.abs(A[good] @ s2 - bo[good]), atol=1e-9)


@pytest.mark.parametrize("case", range(11))
def test_solve_pairs_matches_reference_build(case):
    """The product's host FP64 solve against the reference's own OD_Threshold
    and least-squares steps (mfunc.h, DFAlign.cu:875-948 built with the
    project's SP++ stand-in; fixtures from tests/golden/make_golden.py)."""
    import json
    c = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_solve_cases.json")))[case]
    nf = c["nframe"]
    pairs = np.array(c["pairs"], dtype=np.int32)
    b = np.array(c["b"], dtype=np.float32)
    r = api.solve_pairs(nf, pairs, b, c["kithresh"])
    np.testing.assert_allclose(r["ki1"], c["ki1"], rtol=0, atol=1e-9)
    assert r["kept"].tolist() == c["good"]
    np.testing.assert_allclose(r["ki2"], c["ki2"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(r["step"], np.array(c["shift"]), rtol=0, atol=1e-9)


def test_solve_pairs_rejects_bad_pairs():
    with pytest.raises(_lib.McError):
        api.solve_pairs(4, np.array([[2, 1]]), np.zeros((1, 2)))


def test_schedule_table_host_only():
    api.schedule_clear()
    assert api.schedule_get(3710) is None
    qs = api.schedule_candidates(3710)
    assert 70 in qs and 35 in qs and all(3710 % q == 0 for q in qs)
    api.schedule_set(3710, pair_q=35, pairs_per_cta=16)
    assert api.schedule_get(3710) == {"n": 3710, "pair_q": 35, "pairs_per_cta": 16, "pair_variant": 0,
                                      "fwd_streams": 0, "fwd_rows_pairing": 0, "fwd_cols_pairing": 0}
    api.schedule_set(3710, pair_q=35, fwd_streams=2, fwd_rows_pairing=1, fwd_cols_pairing=2)
    assert api.schedule_get(3710)["fwd_streams"] == 2 and api.schedule_get(3710)["fwd_cols_pairing"] == 2
    api.schedule_set(3710, pair_q=70)
    assert api.schedule_get(3710)["pair_q"] == 70
    with pytest.raises(_lib.McError):
        api.schedule_set(3710, pair_q=3)          # 3710 = 1236.67 * 3: no split
    with pytest.raises(_lib.McError):
        api.schedule_set(3710, pair_q=2)          # P = 1855 above the codelet team size
    with pytest.raises(_lib.McError):
        api.schedule_set(3710, pair_variant=2)
    with pytest.raises(_lib.McError):
        api.schedule_set(3710, fwd_streams=9)
    with pytest.raises(_lib.McError):
        api.schedule_set(3710, fwd_rows_pairing=3)
    api.schedule_clear()
    assert api.schedule_get(3710) is None


def test_batch_requires_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("host-only check")
    with pytest.raises(_lib.McError):
        api.Batch(0, 2)
    L = _lib.lib()
    h = C.c_void_p()
    assert L.mc_batch_create(0, 0, C.byref(h)) == -1   # lanes outside [1, 16]
    assert L.mc_batch_run(None, None, 0, None) == -1
