"""The image sum runs as two kernels for sizes with a two-level transform
(k_shift_acc, then k_sum_cols2l with a transposed store) and as the single
fused k_shift_sum for other sizes.  Both forms, and the raw and partial sums
that share them (-srs, -2es), are checked against the FP64 oracle's
phase-shift-and-sum (DFAlign.cu:1114-1292) at relative L2 <= 1e-5."""
import numpy as np
import pytest

from motioncorr1exp_b200 import api, synth
from oracle import mc_oracle as O

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


# 512 and 1024 take the split kernels (two-level sizes); 500 and 966 the fused one
@pytest.mark.parametrize("crop, nx, ny", [(512, 560, 540), (1024, 1060, 1040), (500, 530, 520), (966, 1000, 990)])
def test_sum_forms_match_oracle(gpu, crop, nx, ny):
    nz = 10
    mv = synth.make_movie(nx, ny, nz, mean=2.0, seed=83, dtype="u8", speed=0.6, rw_sigma=0.4)
    p = api.verify_params(api.Params(crop_nsam=crop, CCPeakSearchDim=64), nz)
    with api.Plan(p, nx, ny, nz, 0) as pl:
        pl.load_frames(mv.frames[pl.info["nstart"]: pl.info["nend"] + 1])
        img = pl.run()
        sh, first, last = pl.sum_shifts()
        raw = pl.raw_sum()
        mid = first + (last - first) // 2
        part = pl.sum_to(mid + pl.info["nstart"])
    assert img.shape == (crop, crop)
    op = O.Params(**{k: getattr(p, k) for k in O.Params.__dataclass_fields__})
    ref = O.align_movie(mv.frames, 0, op, keep_spectra=True)
    F = ref.spectra
    assert rel_l2(img, ref.image) <= 1e-5
    assert rel_l2(raw, O.raw_sum_image(F, first, last)) <= 1e-5
    # the second sum: the corrected sum's shifts over frames first..mid
    S = None
    for k in range(first, mid + 1):
        s = complex(sh[k, 0], sh[k, 1])
        t = F[k] if (k == first and not p.bAlignToMid) else O.phase_shift(F[k], s.real, s.imag)
        S = t if S is None else S + t
    assert rel_l2(part, O.spectrum_to_image(S)) <= 1e-5
