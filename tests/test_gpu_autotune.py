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


def test_forward_schedule_trials_and_pairings(gpu):
    """The forward half of the tuner (forked streams x radix-53 pairing of the
    row and column passes), and every pairing of the 3710 = 53 x 70
    transforms giving the oracle's spectra."""
    import numpy as np
    from motioncorr1exp_b200 import synth
    from oracle import mc_oracle as O
    api.schedule_clear()
    try:
        r = autotune.tune(512, box=64, nframes=8, fod=1, reps=1)
        assert len(r["fwd_trials"]) == len(autotune.FWD_STREAMS) * 4
        # the fastest trial, or the built-in schedule (4 streams, both passes
        # paired) when it is within 1 % of the fastest
        best = min(t["ms"] for t in r["fwd_trials"])
        chosen = next(t for t in r["fwd_trials"] if (t["fwd_streams"], t["fwd_rows_pairing"], t["fwd_cols_pairing"])
                      == (r["fwd_streams"], r["fwd_rows_pairing"], r["fwd_cols_pairing"]))
        assert r["fwd_ms"] == chosen["ms"] > 0
        assert r["fwd_ms"] == best or ((r["fwd_streams"], r["fwd_rows_pairing"], r["fwd_cols_pairing"]) == (4, 2, 2)
                                       and r["fwd_ms"] <= 1.01 * best)
        assert api.schedule_get(512)["fwd_streams"] == r["fwd_streams"]
        mv = synth.make_movie(3838, 3710, 3, mean=1.2, seed=71, dtype="u8")
        o = O.forward_spectrum(O.decode_frame(mv.frames[2], 0), 0, 0, 3710, 3710)
        p = api.verify_params(api.Params(FrameDistOffset=0), 3)
        for rp in (1, 2):
            for cp in (1, 2):
                api.schedule_set(3710, pair_q=70, pairs_per_cta=32, fwd_streams=2, fwd_rows_pairing=rp,
                                 fwd_cols_pairing=cp)
                with api.Plan(p, 3838, 3710, 3, 0) as pl:
                    pl.load_frames(mv.frames)
                    pl.forward()
                    g = pl.spectrum(2)
                assert np.linalg.norm(g - o) / np.linalg.norm(o) <= 1e-5, (rp, cp)
    finally:
        api.schedule_clear()
