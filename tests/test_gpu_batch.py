"""Batching: plan re-targeting (mc_plan_reframe), in-place device frames
(mc_plan_bind_frames_device), pair-stage schedules and the multi-lane batch
runner (mc_batch_run) against one-at-a-time plans."""
import numpy as np
import pytest
import torch

from motioncorr1exp_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu


def _one(mv, params, mode=0):
    nz, ny, nx = mv.frames.shape
    with api.Plan(params, nx, ny, nz, mode) as pl:
        fr = mv.frames[pl.info["nstart"]: pl.info["nend"] + 1]
        pl.load_frames(fr)
        img = pl.run()
        return img, pl.frame_shifts().copy(), pl.pair_results()


def _movie(nx, ny, nz, seed):
    return synth.make_movie(nx, ny, nz, mean=1.5, seed=seed, dtype="u8", speed=0.4, rw_sigma=0.5)


def test_reframe_matches_fresh_plans(gpu):
    a = _movie(300, 290, 14, 41)
    b = _movie(300, 290, 9, 42)
    pa = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=2), 14)
    pb = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=1, kiThresh=0.3, nStart=1), 9)
    ref_a = _one(a, pa)
    ref_b = _one(b, pb)
    with api.Plan(pa, 300, 290, 14, 0, cap_frames=16, cap_pairs=80) as pl:
        for mv, p, ref in ((a, pa, ref_a), (b, pb, ref_b), (a, pa, ref_a)):
            pl.reframe(p, mv.frames.shape[0])
            pl.load_frames(mv.frames[pl.info["nstart"]: pl.info["nend"] + 1])
            img = pl.run()
            np.testing.assert_array_equal(img, ref[0])
            np.testing.assert_array_equal(pl.frame_shifts(), ref[1])
            for k in ("pairs", "shift", "peak"):
                np.testing.assert_array_equal(pl.pair_results()[k], ref[2][k])
        # beyond the capacity
        big = api.verify_params(api.Params(CCPeakSearchDim=64), 20)
        with pytest.raises(_lib.McError):
            pl.reframe(big, 20)
        # another geometry
        with pytest.raises(_lib.McError):
            pl.reframe(api.verify_params(api.Params(CCPeakSearchDim=32), 14), 14)


def test_bound_device_frames_match_loaded(gpu):
    mv = _movie(256, 256, 10, 43)
    p = api.verify_params(api.Params(CCPeakSearchDim=64), 10)
    ref = _one(mv, p)
    d = torch.from_numpy(mv.frames).cuda()
    with api.Plan(p, 256, 256, 10, 0) as pl:
        for _ in range(2):       # capture, then replay with the bound pointer
            pl.bind_frames_device(d.data_ptr())
            img = pl.run()
            np.testing.assert_array_equal(img, ref[0])
            np.testing.assert_array_equal(pl.frame_shifts(), ref[1])
        pl.bind_frames_device(0)
        with pytest.raises(_lib.McError):
            pl.run()             # nothing loaded after unbinding
        with pytest.raises(_lib.McError):
            pl.bind_frames_device(mv.frames.ctypes.data)   # host memory


def test_schedule_changes_split_and_keeps_results(gpu):
    mv = _movie(256, 256, 10, 44)
    p = api.verify_params(api.Params(CCPeakSearchDim=64), 10)
    with api.Plan(p, 256, 256, 10, 0) as pl:
        n = pl.nsam
        q0 = pl.info["prune_q"]
    ref = _one(mv, p)
    alt = [q for q in api.schedule_candidates(n) if q != q0]
    assert len(alt) >= 2          # 256 = 64*4 = 32*8 = 16*16 = 8*32 = 4*64
    try:
        api.schedule_set(n, pair_q=alt[0], pairs_per_cta=8)
        with api.Plan(p, 256, 256, 10, 0) as pl:
            assert pl.info["prune_q"] == alt[0]
            pl.load_frames(mv.frames)
            img = pl.run()
            np.testing.assert_allclose(pl.frame_shifts(), ref[1], rtol=0, atol=0.01)
            np.testing.assert_array_equal(pl.pair_results()["peak"], ref[2]["peak"])
            rel = np.linalg.norm(img - ref[0]) / np.linalg.norm(ref[0])
            assert rel < 1e-5
    finally:
        api.schedule_clear()


@pytest.mark.parametrize("lanes,on_device", [(1, False), (3, False), (3, True)])
def test_batch_matches_one_at_a_time(gpu, lanes, on_device):
    rng = np.random.default_rng(45)
    geos = [(256, 256), (300, 290), (320, 320)]
    movies, refs, keep = [], [], []
    for i in range(7):
        nx, ny = geos[i % 3]
        nz = int(rng.integers(6, 15))
        fod = int(rng.choice([1, 2]))
        if nz // 2 - fod < 1:
            fod = 0
        mv = _movie(nx, ny, nz, 100 + i)
        p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=fod), nz)
        refs.append(_one(mv, p))
        ns, ne = p.nStart, min(p.nEnd, nz - 1)
        fr = np.ascontiguousarray(mv.frames[ns: ne + 1])
        n = refs[-1][0].shape[0]
        m = {"params": p, "nx": nx, "ny": ny, "nz": nz, "mode": 0,
             "image": np.zeros((n, n), np.float32), "frame_shifts": np.zeros((ne - ns + 1, 2))}
        if on_device:
            d = torch.from_numpy(fr).cuda()
            keep.append(d)
            m["device_ptr"] = d.data_ptr()
        else:
            m["frames"] = fr
        movies.append(m)
    with api.Batch(0, lanes) as b:
        for _ in range(2):               # second run reuses plans and graphs
            out = b.run(movies)
            for m, r, ref in zip(movies, out, refs):
                assert r["status"] == 0 and r["nframe"] == m["frame_shifts"].shape[0]
                assert r["end_ms"] >= r["start_ms"] and r["gpu_ms"] > 0
                np.testing.assert_array_equal(m["image"], ref[0])
                np.testing.assert_array_equal(m["frame_shifts"], ref[1])
        assert {r["lane"] for r in out} <= set(range(lanes))
        assert b.device_bytes > 0


def test_batch_reports_failing_movie(gpu):
    mv = _movie(256, 256, 8, 46)
    p = api.verify_params(api.Params(CCPeakSearchDim=64), 8)
    bad = api.Params(**{**p.__dict__, "GPUNum": 7})
    img = np.zeros((256, 256), np.float32)
    movies = [{"params": p, "nx": 256, "ny": 256, "nz": 8, "mode": 0, "frames": mv.frames, "image": img},
              {"params": bad, "nx": 256, "ny": 256, "nz": 8, "mode": 0, "frames": mv.frames}]
    with api.Batch(0, 2) as b:
        out = b.run(movies, check=False)
        assert out[0]["status"] == 0 and out[1]["status"] == -1
        assert "GPUNum" in out[1]["message"]
        np.testing.assert_array_equal(img, _one(mv, p)[0])
        with pytest.raises(_lib.McError):
            b.run(movies)


def test_graph_serves_every_bound_buffer(gpu):
    """One captured movie graph, frame buffers swapped between replays: the
    frame base is read on the device, so each replay aligns the bound movie."""
    a, b = _movie(256, 256, 10, 47), _movie(256, 256, 10, 48)
    p = api.verify_params(api.Params(CCPeakSearchDim=64), 10)
    ref_a, ref_b = _one(a, p), _one(b, p)
    da, db = torch.from_numpy(a.frames).cuda(), torch.from_numpy(b.frames).cuda()
    with api.Plan(p, 256, 256, 10, 0) as pl:
        for d, ref in ((da, ref_a), (db, ref_b), (da, ref_a), (db, ref_b)):
            pl.bind_frames_device(d.data_ptr())
            img = pl.run()
            np.testing.assert_array_equal(img, ref[0])
            np.testing.assert_array_equal(pl.frame_shifts(), ref[1])
        # the plan's own buffer after bound ones
        pl.load_frames(a.frames)
        np.testing.assert_array_equal(pl.run(), ref_a[0])


def _build_stress(tmp_path, libdir, extra=()):
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "batch_stress")
    subprocess.run(["g++", "-O1", "-g", "-std=c++17", *extra, "-I", os.path.join(root, "include"),
                    "-I", "/usr/local/cuda/include", os.path.join(root, "tests", "native", "batch_stress.cpp"),
                    "-L", libdir, "-lmc", "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{libdir}",
                    "-o", exe], check=True, capture_output=True)
    return exe


def test_batch_stress_native(gpu, tmp_path):
    """Three lanes, 30 movies of three geometries and two pixel types, frames
    in device, pinned and pageable host memory, three rounds (plans
    re-targeted, graphs replayed, the queue reversed): every image and shift
    list bit-identical to a fresh one-at-a-time plan."""
    import os
    import subprocess
    exe = _build_stress(tmp_path, os.path.dirname(_lib.LIB_PATH))
    r = subprocess.run([exe, "3", "30", "3"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 mismatches" in r.stdout


def _graph_movies(seed, count, geos=((256, 256), (300, 290), (320, 320))):
    rng = np.random.default_rng(seed)
    movies, refs, keep = [], [], []
    for i in range(count):
        nx, ny = geos[i % len(geos)]
        nz = int(rng.integers(6, 15))
        fod = int(rng.choice([1, 2]))
        if nz // 2 - fod < 1:
            fod = 0
        mv = _movie(nx, ny, nz, seed + i)
        p = api.verify_params(api.Params(CCPeakSearchDim=64, FrameDistOffset=fod), nz)
        refs.append(_one(mv, p))
        d = torch.from_numpy(np.ascontiguousarray(mv.frames)).cuda()
        keep.append(d)
        n = refs[-1][0].shape[0]
        img = torch.zeros((n, n), dtype=torch.float32, pin_memory=True)
        keep.append(img)
        movies.append({"params": p, "nx": nx, "ny": ny, "nz": nz, "mode": 0, "device_ptr": d.data_ptr(),
                       "image": img.numpy(), "frame_shifts": np.zeros((nz, 2))})
    return movies, refs, keep


@pytest.mark.parametrize("lanes", [1, 2, 3])
def test_batch_single_graph_matches_one_at_a_time(gpu, lanes):
    """Single-graph mode: the whole batch captured as one CUDA graph (lanes as
    branches), launched once per run and relaunched while the job list stays
    the same; another job list is captured anew.  Every image and shift list
    bit-identical to a fresh one-at-a-time plan."""
    movies, refs, keep = _graph_movies(200, 8)
    with api.Batch(0, lanes, graph=True) as b:
        for sub in (movies, movies, movies[2:7], movies):
            for m in sub:
                m["image"][:] = -1.0
                m["frame_shifts"][:] = -1.0
            out = b.run(sub)
            for m, r in zip(sub, out):
                ref = refs[next(k for k, x in enumerate(movies) if x is m)]
                assert r["status"] == 0 and r["nframe"] == m["frame_shifts"].shape[0]
                np.testing.assert_array_equal(m["image"], ref[0])
                np.testing.assert_array_equal(m["frame_shifts"], ref[1])
        # the same plans then serve the threaded mode
        b2 = api.Batch(0, lanes)
        out = b2.run(movies)
        b2.close()
        for m, ref in zip(movies, refs):
            np.testing.assert_array_equal(m["image"], ref[0])


def test_batch_single_graph_rejects(gpu):
    movies, refs, keep = _graph_movies(300, 2)
    with api.Batch(0, 2, graph=True) as b:
        host = dict(movies[0])
        del host["device_ptr"]
        host["frames"] = np.zeros((host["nz"], host["ny"], host["nx"]), np.uint8)
        with pytest.raises(_lib.McError, match="device memory"):
            b.run([host])
        itr = dict(movies[0], params=api.Params(**{**movies[0]["params"].__dict__, "iter": 2}))
        with pytest.raises(_lib.McError, match="device-only"):
            b.run([itr])
        pageable = dict(movies[1], image=np.zeros_like(movies[1]["image"]))
        with pytest.raises(_lib.McError, match="pinned"):
            b.run([pageable])
        out = b.run(movies)              # and it still runs the valid list
        for m, ref in zip(movies, refs):
            np.testing.assert_array_equal(m["image"], ref[0])
