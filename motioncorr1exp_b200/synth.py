"""Seeded synthetic dose-fractionated movies.

Signal model (one canvas per movie, shifted per frame):
  * white Gaussian noise low-pass filtered at 0.1 cycles/px, normalised to
    unit standard deviation;
  * plus Gaussian blobs (sigma 6 px, amplitude 2), 200 per 1024^2 of frame
    area;
  * the canvas is padded by at least 64 px beyond the largest drift and every
    frame is a Fourier (sub-pixel) shift of it, cropped to nx x ny, so the
    periodic wrap of the shift never reaches the crop;
  * per-pixel rate = mean * max(0, 1 + 0.5 * signal), counts ~ Poisson(rate).

Drift models: ``linear`` (v px/frame + random walk), ``jitter`` (random walk
+ sinusoid).  ``truth[k]`` is the displacement (dx, dy) of frame k's content
relative to the canvas: frame_k(x) = canvas(x - truth[k]).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

try:
    import scipy.fft as _fft

    def _rfft2(a):
        return _fft.rfft2(a, workers=-1)

    def _irfft2(a, s):
        return _fft.irfft2(a, s=s, workers=-1)
except Exception:  # pragma: no cover
    def _rfft2(a):
        return np.fft.rfft2(a)

    def _irfft2(a, s):
        return np.fft.irfft2(a, s=s)


@dataclass
class Movie:
    frames: np.ndarray      # (nz, ny, nx) uint8 (MRC mode 0 bytes) or float32 (mode 2)
    mode: int               # MRC mode the frames are stored in
    truth: np.ndarray       # (nz, 2) float64 displacement of frame content
    seed: int


def drift_track(nframes: int, rng: np.random.Generator, kind: str = "linear",
                speed: float = 0.4, rw_sigma: float = 0.3, amp: float = 1.5,
                period: float = 20.0) -> np.ndarray:
    """Ground-truth displacement per frame, frame 0 at the origin."""
    theta = rng.uniform(0.0, 2.0 * math.pi)
    direction = np.array([math.cos(theta), math.sin(theta)])
    steps = rng.normal(0.0, rw_sigma, size=(nframes, 2))
    steps[0] = 0.0
    walk = np.cumsum(steps, axis=0)
    k = np.arange(nframes)[:, None]
    if kind == "linear":
        det = speed * k * direction[None, :]
    elif kind == "jitter":
        det = amp * np.sin(2.0 * math.pi * k / period) * direction[None, :]
    else:
        raise ValueError(f"unknown drift kind {kind!r}")
    track = walk + det
    return track - track[0]


def signal_canvas(cy: int, cx: int, rng: np.random.Generator, area_px: int,
                  cutoff: float = 0.1, blob_sigma: float = 6.0, blob_amp: float = 2.0,
                  blobs_per_mpx: float = 200.0) -> np.ndarray:
    """Low-passed unit-variance noise plus Gaussian blobs on a cy x cx canvas."""
    noise = rng.standard_normal((cy, cx)).astype(np.float32)
    F = _rfft2(noise)
    fy = np.fft.fftfreq(cy)[:, None]
    fx = np.fft.rfftfreq(cx)[None, :]
    F[(fy * fy + fx * fx) > cutoff * cutoff] = 0
    s = _irfft2(F, s=(cy, cx)).astype(np.float32)
    s /= max(float(s.std()), 1e-12)
    nblob = int(round(blobs_per_mpx * area_px / (1024.0 * 1024.0)))
    r = int(math.ceil(4 * blob_sigma))
    g = np.arange(-r, r + 1, dtype=np.float32)
    for _ in range(nblob):
        y0 = rng.uniform(0, cy)
        x0 = rng.uniform(0, cx)
        iy, ix = int(y0), int(x0)
        wy = np.exp(-0.5 * ((g + iy - y0) / blob_sigma) ** 2)
        wx = np.exp(-0.5 * ((g + ix - x0) / blob_sigma) ** 2)
        ys = slice(max(iy - r, 0), min(iy + r + 1, cy))
        xs = slice(max(ix - r, 0), min(ix + r + 1, cx))
        wy = wy[ys.start - (iy - r): ys.stop - (iy - r)]
        wx = wx[xs.start - (ix - r): xs.stop - (ix - r)]
        s[ys, xs] += blob_amp * wy[:, None] * wx[None, :]
    return s


def make_movie(nx: int, ny: int, nframes: int, mean: float, seed: int,
               dtype: str = "u8", kind: str = "linear", speed: float = 0.4,
               rw_sigma: float = 0.3, amp: float = 1.5, period: float = 20.0,
               contrast: float = 0.5) -> Movie:
    """Seeded Poisson movie.  ``dtype`` 'u8' -> MRC mode 0 bytes, 'f32' -> mode 2."""
    rng = np.random.Generator(np.random.PCG64(seed))
    truth = drift_track(nframes, rng, kind, speed, rw_sigma, amp, period)
    pad = 64 + int(math.ceil(np.abs(truth).max() if nframes else 0.0))
    cy, cx = ny + 2 * pad, nx + 2 * pad
    canvas = signal_canvas(cy, cx, rng, nx * ny)
    C = _rfft2(canvas)
    fy = np.fft.fftfreq(cy)[:, None]
    fx = np.fft.rfftfreq(cx)[None, :]
    out = np.empty((nframes, ny, nx), dtype=np.uint8 if dtype == "u8" else np.float32)
    for k in range(nframes):
        dx, dy = truth[k]
        ph = np.exp(-2j * math.pi * (fx * dx + fy * dy)).astype(np.complex64)
        img = _irfft2(C * ph, s=(cy, cx))[pad:pad + ny, pad:pad + nx]
        rate = mean * np.maximum(0.0, 1.0 + contrast * img)
        counts = rng.poisson(rate)
        if dtype == "u8":
            if counts.max(initial=0) > 127:
                raise ValueError("counts above 127 do not survive MRC mode 0 (signed char)")
            out[k] = counts.astype(np.uint8)
        else:
            out[k] = counts.astype(np.float32)
    return Movie(frames=out, mode=0 if dtype == "u8" else 2, truth=truth, seed=seed)


def make_movie_torch(nx: int, ny: int, nframes: int, mean: float, seed: int, dtype: str = "u8",
                     kind: str = "linear", speed: float = 0.4, rw_sigma: float = 0.3, amp: float = 1.5,
                     period: float = 20.0, contrast: float = 0.5, device: str = "cuda"):
    """Same signal model generated with torch on ``device`` (fast full-size
    inputs).  Blobs are deposited on integer pixels and blurred in Fourier
    space.  Returns (frames tensor (nz, ny, nx) uint8|float32 on device, truth)
    after the device has finished writing them."""
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    truth = drift_track(nframes, rng, kind, speed, rw_sigma, amp, period)
    pad = 64 + int(math.ceil(np.abs(truth).max() if nframes else 0.0))
    cy, cx = ny + 2 * pad, nx + 2 * pad
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    fy = torch.fft.fftfreq(cy, device=device)[:, None]
    fx = torch.fft.rfftfreq(cx, device=device)[None, :]
    f2 = fy * fy + fx * fx
    noise = torch.randn((cy, cx), generator=g, device=device)
    F = torch.fft.rfft2(noise)
    F = F * (f2 <= 0.01)
    s = torch.fft.irfft2(F, s=(cy, cx))
    s = s / s.std().clamp_min(1e-12)
    nblob = int(round(200.0 * nx * ny / (1024.0 * 1024.0)))
    pos = torch.randint(0, cy * cx, (nblob,), generator=g, device=device)
    dep = torch.zeros(cy * cx, device=device)
    dep.index_add_(0, pos, torch.full((nblob,), 2.0, device=device))
    blob = torch.fft.irfft2(torch.fft.rfft2(dep.view(cy, cx)) * torch.exp(-2.0 * math.pi ** 2 * 36.0 * f2),
                            s=(cy, cx))
    C = torch.fft.rfft2(s + blob)
    out = torch.empty((nframes, ny, nx), dtype=torch.uint8 if dtype == "u8" else torch.float32, device=device)
    for k in range(nframes):
        dx, dy = (float(v) for v in truth[k])
        ph = torch.exp(-2j * math.pi * (fx * dx + fy * dy))
        img = torch.fft.irfft2(C * ph, s=(cy, cx))[pad:pad + ny, pad:pad + nx]
        rate = mean * torch.clamp(1.0 + contrast * img, min=0.0)
        counts = torch.poisson(rate, generator=g)
        out[k] = counts.clamp(max=127).to(out.dtype) if dtype == "u8" else counts.to(out.dtype)
    # the frames are complete before they are returned: libmc's plans copy or
    # read them on their own non-blocking streams, which do not wait for
    # torch's stream
    torch.cuda.synchronize(out.device)
    return out, truth


# Named workloads: frames, size, dtype, dose, drift and flags of each benchmark form.
WORKLOADS = {
    "c1": dict(nx=1024, ny=1024, nframes=16, mean=1.5, dtype="f32", kind="linear",
               speed=0.4, rw_sigma=0.3, flags=dict(bin=1.0, FrameDistOffset=2, bfactor=150.0,
                                                  CCPeakSearchDim=96, NoisePeakSize=0)),
    "c2": dict(nx=3838, ny=3710, nframes=40, mean=1.2, dtype="u8", kind="linear",
               speed=0.3, rw_sigma=0.5, flags=dict(bin=1.0, FrameDistOffset=7, bfactor=150.0,
                                                  CCPeakSearchDim=96, bAlignToMid=1)),
    "c3": dict(nx=7676, ny=7420, nframes=50, mean=0.3, dtype="u8", kind="linear",
               speed=0.3, rw_sigma=0.5, flags=dict(bin=2.0)),
    "c4": dict(nx=4096, ny=4096, nframes=60, mean=1.0, dtype="f32", kind="jitter",
               rw_sigma=0.8, amp=1.5, period=20.0, flags=dict(iter=3, iterthres=0.01)),
}


def make_workload(name: str, seed: int = 0, nframes: int | None = None,
                  scale: int = 1) -> tuple[Movie, dict]:
    """Build one named workload (optionally fewer frames / a 1/scale size)."""
    w = dict(WORKLOADS[name])
    flags = w.pop("flags")
    if nframes is not None:
        w["nframes"] = nframes
    if scale != 1:
        w["nx"] //= scale
        w["ny"] //= scale
    return make_movie(seed=seed, **w), flags


# Batch workload: movies of three sizes, uneven depth and pair distance.
C5_GEOMETRIES = [(2048, 2048), (3838, 3710), (4096, 4096)]


def c5_jobs(seed: int = 0, n_movies: int = 32, max_frames: int = 80) -> tuple[list[dict], list[float]]:
    """Job list of the batch workload: per movie a geometry from
    C5_GEOMETRIES, F ~ U[20, max_frames] frames, fod in {2, 4, 7} and a
    window [offset, offset + F) of that geometry's base movie (max_frames
    frames, mean dose U[0.8, 1.5] e/px/frame, returned per geometry)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    means = [float(rng.uniform(0.8, 1.5)) for _ in C5_GEOMETRIES]
    jobs = []
    for _ in range(n_movies):
        g = int(rng.integers(0, len(C5_GEOMETRIES)))
        nf = int(rng.integers(20, max_frames + 1))
        fod = int(rng.choice([2, 4, 7]))
        off = int(rng.integers(0, max_frames - nf + 1))
        nx, ny = C5_GEOMETRIES[g]
        jobs.append(dict(geometry=g, nx=nx, ny=ny, nframes=nf, fod=fod, offset=off))
    return jobs, means
