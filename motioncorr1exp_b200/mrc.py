"""MRC stack reader/writer with the header layout of the reference.

The 1024-byte header follows ``struct MRCHeader`` (mrcheader.h:3-45).  Frame
``n`` starts at 1024 + nsymbt + n * nx*ny*wordlength (MRC::read2DIm,
mrc.cpp:151-157).  ``write_image`` produces the same bytes as
``MRC::createMRC(float*)`` (mrc.cpp:243-274): mode 2, cellb 90/90/90, axes
1/2/3, dmin/dmax from a float scan, dmean accumulated in double, and no
``MAP `` stamp.
"""
from __future__ import annotations

import os

import numpy as np

HEADER_DTYPE = np.dtype([
    ("nx", "<i4"), ("ny", "<i4"), ("nz", "<i4"), ("mode", "<i4"),
    ("nxstart", "<i4"), ("nystart", "<i4"), ("nzstart", "<i4"),
    ("mx", "<i4"), ("my", "<i4"), ("mz", "<i4"),
    ("cella", "<f4", 3), ("cellb", "<f4", 3),
    ("mapc", "<i4"), ("mapr", "<i4"), ("maps", "<i4"),
    ("dmin", "<f4"), ("dmax", "<f4"), ("dmean", "<f4"),
    ("ispg", "<i4"), ("nsymbt", "<i4"),
    ("extra", "V100"),
    ("origin", "<f4", 3),
    ("map", "S4"), ("machst", "<i4"), ("rms", "<f4"), ("nlabels", "<i4"),
    ("label", "S80", 10),
])
assert HEADER_DTYPE.itemsize == 1024

# MRC::getWordLength (mrc.cpp:99-118)
WORD_LENGTH = {0: 1, 1: 2, 2: 4, 3: 4, 4: 8, 6: 2, 12: 2}
PIXEL_DTYPE = {0: np.int8, 1: np.int16, 2: np.float32, 6: np.uint16, 12: np.float16}  # 12: MRC2014 half


def default_header() -> np.ndarray:
    """The MRC() constructor's header (mrc.cpp:5-16)."""
    h = np.zeros((), dtype=HEADER_DTYPE)
    h["mode"] = 2
    h["cellb"] = (90, 90, 90)
    h["mapc"], h["mapr"], h["maps"] = 1, 2, 3
    return h


def read_header(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        raw = f.read(1024)
    if len(raw) < 1024:
        raise ValueError(f"{path}: shorter than an MRC header")
    return np.frombuffer(raw, dtype=HEADER_DTYPE)[0].copy()


def read_stack(path: str, first: int = 0, count: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Raw frames (count, ny, nx) in the file's pixel type, plus the header."""
    h = read_header(path)
    nx, ny, nz, mode = int(h["nx"]), int(h["ny"]), int(h["nz"]), int(h["mode"])
    if mode not in PIXEL_DTYPE:
        raise ValueError(f"{path}: unsupported MRC mode {mode}")
    if count is None:
        count = nz - first
    im = nx * ny * WORD_LENGTH[mode]
    off = 1024 + int(h["nsymbt"]) + first * im
    need = off + count * im
    if os.path.getsize(path) < need:
        raise ValueError(f"{path}: truncated ({os.path.getsize(path)} < {need} bytes)")
    data = np.fromfile(path, dtype=PIXEL_DTYPE[mode], count=count * nx * ny, offset=off)
    return data.reshape(count, ny, nx), h


def write_stack(path: str, frames: np.ndarray, mode: int) -> None:
    """Write raw frames with a header that says ``mode`` (tests, synthetic data)."""
    frames = np.ascontiguousarray(frames)
    nz, ny, nx = frames.shape
    h = default_header()
    h["nx"], h["ny"], h["nz"], h["mode"] = nx, ny, nz, mode
    h["map"] = b"MAP "
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(frames.astype(PIXEL_DTYPE[mode], copy=False).tobytes())


def image_header(data: np.ndarray) -> np.ndarray:
    """Header createMRC(float*) writes for ``data`` (mrc.cpp:243-268)."""
    d = np.asarray(data, dtype=np.float32)
    nz = 1 if d.ndim == 2 else d.shape[0]
    ny, nx = d.shape[-2], d.shape[-1]
    h = default_header()
    h["nx"], h["ny"], h["nz"], h["mode"] = nx, ny, nz, 2
    flat = d.ravel()
    h["dmin"] = flat.min() if flat.size else 0
    h["dmax"] = flat.max() if flat.size else 0
    # mean is accumulated in double in element order, then stored as float
    h["dmean"] = np.float32(np.add.accumulate(flat.astype(np.float64))[-1] / flat.size) if flat.size else 0
    return h


def write_image(path: str, data: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(data, dtype=np.float32)
    h = image_header(d)
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(d.tobytes())
    return h


def read_image(path: str) -> np.ndarray:
    frames, _ = read_stack(path)
    return frames[0] if frames.shape[0] == 1 else frames
