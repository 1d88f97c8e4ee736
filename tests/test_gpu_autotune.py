"""Autotuner: every trial runs, the winner is installed, the JSON cache
round-trips and plans created afterwards use the cached split."""
import json

import pytest

from motioncorr1exp_b200 import api, autotune

pytestmark = pytest.mark.gpu


def test_tune_save_load(gpu, tmp_path):
    api.schedule_clear()
    try:
        r = autotune.tune(512, box=64, nframes=8, fod=1, reps=1)
        qs = api.schedule_candidates(512)
        assert {t["pair_q"] for t in r["trials"]} == set(qs)
        assert len(r["trials"]) == len(qs) * len(autotune.PAIRS_PER_CTA)
        assert r["ms"] == min(t["ms"] for t in r["trials"]) > 0
        path = str(tmp_path / "s.json")
        autotune.save({512: r}, "test-gpu", path)
        data = json.load(open(path))
        assert data["test-gpu"]["512"]["pair_q"] == r["pair_q"]
        api.schedule_clear()
        assert autotune.load(path, gpu="test-gpu") == 1
        assert api.schedule_get(512)["pair_q"] == r["pair_q"]
        p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=1), 8)
        with api.Plan(p, 512, 512, 8, 0) as pl:
            assert pl.info["prune_q"] == r["pair_q"]
        assert autotune.load(path, gpu="other-gpu") == 0
    finally:
        api.schedule_clear()
