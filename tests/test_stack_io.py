"""Stack files through mc_stack_* (host only, no GPU): MRC, MRC-gz and strip
TIFF with the detection order of the alignment thread (DFAlign.cu:470-479).

TIFF decodes are checked against PIL's bundled libtiff (the library MRCT
calls, mrct.cpp:113-152) on files libtiff itself wrote: none, LZW (with and
without predictor 2, with table resets), Deflate, PackBits, several strips.
BigTIFF, big-endian words and the rejected variants use the small writer
below, which follows the TIFF 6.0 / BigTIFF layouts."""
import gzip
import struct
import zlib

import numpy as np
import pytest

from motioncorr1exp_b200 import _lib, api, mrc

PIL = pytest.importorskip("PIL.Image")


def pil_frames(path):
    im = PIL.open(path)
    out = []
    for i in range(im.n_frames):
        im.seek(i)
        out.append(np.array(im))
    return np.array(out)


def pil_write(path, frames, **kw):
    ims = [PIL.fromarray(f) for f in frames]
    ims[0].save(path, save_all=True, append_images=ims[1:], **kw)


def write_tiff(path, frames, *, be=False, big=False, rps=None, compression=1, predictor=1, bits=None,
               extra=()):
    """Strip TIFF writer: one directory per frame, values of `frames` stored
    as unsigned words in the chosen byte order (predictor 2 differences
    taken on the words, then swapped), Deflate via zlib."""
    e = ">" if be else "<"
    nz, ny, nx = frames.shape
    wb = frames.dtype.itemsize
    bps = 8 * wb if bits is None else bits
    rps = rps or ny
    out = bytearray(b"MM" if be else b"II")
    if big:
        out += struct.pack(e + "HHHQ", 43, 8, 0, 0)
        link = 8
    else:
        out += struct.pack(e + "HI", 42, 0)
        link = 4
    off_type, cnt_fmt, val_bytes = (16, "Q", 8) if big else (4, "I", 4)
    fmt = {3: "H", 4: "I", 16: "Q"}
    for f in frames:
        w = f.astype(np.uint16 if wb == 2 else np.uint8)
        if predictor == 2:
            w = w.copy()
            w[:, 1:] = (w[:, 1:].astype(np.int64) - w[:, :-1].astype(np.int64)) % (1 << (8 * wb))
        raw = w.astype(w.dtype.newbyteorder(e)).tobytes()
        offs, cnts = [], []
        for r in range(0, ny, rps):
            chunk = raw[r * nx * wb:(r + rps) * nx * wb]
            if compression == 8:
                chunk = zlib.compress(chunk)
            offs.append(len(out))
            cnts.append(len(chunk))
            out += chunk
            if len(out) % 2:
                out += b"\0"
        tags = sorted([(256, 4, [nx]), (257, 4, [ny]), (258, 3, [bps]), (259, 3, [compression]),
                       (262, 3, [1]), (273, off_type, offs), (277, 3, [1]), (278, 4, [rps]), (279, off_type, cnts),
                       (317, 3, [predictor])] + list(extra))
        entries = []
        for tag, typ, vals in tags:
            data = b"".join(struct.pack(e + fmt[typ], v) for v in vals)
            if len(data) <= val_bytes:
                field = data.ljust(val_bytes, b"\0")
            else:
                field = struct.pack(e + cnt_fmt, len(out))
                out += data
                if len(out) % 2:
                    out += b"\0"
            entries.append(struct.pack(e + "HH" + cnt_fmt, tag, typ, len(vals)) + field)
        ifd = len(out)
        out[link:link + val_bytes] = struct.pack(e + cnt_fmt, ifd)
        out += struct.pack(e + ("Q" if big else "H"), len(entries)) + b"".join(entries)
        link = len(out)
        out += b"\0" * val_bytes
    with open(path, "wb") as fh:
        fh.write(bytes(out))


def rng_frames(seed, shape, dtype, hi):
    return np.random.default_rng(seed).integers(0, hi, shape).astype(dtype)


def smooth_frames(seed, shape, dtype, scale):
    """Low-entropy frames (long LZW strings, the code-equals-next case)."""
    nz, ny, nx = shape
    y, x = np.mgrid[0:ny, 0:nx]
    base = ((x // 7 + y // 5) % 4) * scale
    noise = np.random.default_rng(seed).integers(0, 2, shape)
    return (base[None] + noise).astype(dtype)


@pytest.mark.parametrize("dtype,hi", [(np.uint8, 256), (np.uint16, 65536)])
@pytest.mark.parametrize("kw", [dict(compression=None), dict(compression="tiff_lzw"),
                                dict(compression="tiff_lzw", tiffinfo={317: 2}),
                                dict(compression="tiff_adobe_deflate"), dict(compression="packbits"),
                                dict(compression="tiff_lzw", strip_size=2000)])
def test_tiff_matches_libtiff(tmp_path, dtype, hi, kw):
    for k, frames in enumerate([rng_frames(1, (3, 61, 83), dtype, hi), smooth_frames(2, (3, 61, 83), dtype, 3)]):
        p = str(tmp_path / f"m{k}.tif")
        pil_write(p, frames, **kw)
        want = pil_frames(p)
        np.testing.assert_array_equal(want, frames)
        with api.Stack(p) as s:
            assert (s.nx, s.ny, s.nz) == (83, 61, 3)
            assert s.mode == (api.MODE_U8 if dtype == np.uint8 else 6)
            assert s.info["file_mode"] == 7199 and s.info["format_name"] == "tiff"
            assert s.info["bits"] == 8 * np.dtype(dtype).itemsize
            np.testing.assert_array_equal(s.read_frames(), want)
            np.testing.assert_array_equal(s.read_frames(1, 1)[0], want[1])
            np.testing.assert_array_equal(s.read_frame_float(2), want[2].astype(np.float32))


def test_tiff_lzw_table_resets(tmp_path):
    """A 300 x 257 random frame needs far more than 4094 codes: the encoder
    clears the table mid-strip and the decoder must follow it."""
    frames = rng_frames(3, (2, 257, 300), np.uint8, 256)
    p = str(tmp_path / "big.tif")
    pil_write(p, frames, compression="tiff_lzw")
    with api.Stack(p) as s:
        np.testing.assert_array_equal(s.read_frames(), pil_frames(p))


@pytest.mark.parametrize("be", [False, True])
@pytest.mark.parametrize("big", [False, True])
@pytest.mark.parametrize("compression,predictor", [(1, 1), (8, 1), (8, 2)])
def test_tiff_layouts(tmp_path, be, big, compression, predictor):
    for dtype, hi in [(np.uint8, 256), (np.uint16, 65536)]:
        frames = rng_frames(4, (4, 23, 31), dtype, hi)
        p = str(tmp_path / f"t{np.dtype(dtype).itemsize}.tif")
        write_tiff(p, frames, be=be, big=big, rps=5, compression=compression, predictor=predictor)
        if not big:
            np.testing.assert_array_equal(pil_frames(p), frames)  # libtiff agrees with the writer
        with api.Stack(p) as s:
            assert s.nz == 4 and s.info["compression"] == compression
            np.testing.assert_array_equal(s.read_frames(), frames)


@pytest.mark.parametrize("case,msg", [
    (dict(bits=32), "Only 8-bit or 16-bit TIFF is supported"),
    (dict(extra=[(322, 3, [16]), (323, 3, [16])]), "tiled"),
    (dict(compression=7), "compression 7"),
    (dict(predictor=3), "predictor"),
])
def test_tiff_rejected(tmp_path, case, msg):
    p = str(tmp_path / "bad.tif")
    write_tiff(p, rng_frames(5, (2, 8, 8), np.uint8, 256), **case)
    with pytest.raises(_lib.McError) as ei:
        api.Stack(p)
    assert ei.value.code == -7 and msg in str(ei.value)


def test_tiff_corrupt_strip_reports_frame(tmp_path):
    import ctypes as C
    frames = rng_frames(6, (3, 40, 40), np.uint8, 256)
    p = tmp_path / "c.tif"
    write_tiff(str(p), frames, compression=8)
    b = bytearray(p.read_bytes())
    start = bytes(b).find(zlib.compress(frames[1].tobytes()))
    assert start > 0
    b[start + 2:start + 40] = b"\xff" * 38
    p.write_bytes(bytes(b))
    with api.Stack(str(p)) as s:
        np.testing.assert_array_equal(s.read_frames(0, 1)[0], frames[0])
        out = np.empty((3, 40, 40), np.uint8)
        got = C.c_int()
        rc = s._lib.mc_stack_read_frames(s._h, C.c_void_p(out.ctypes.data), 0, 3, C.byref(got))
        assert rc == -7 and got.value == 1
        assert "frame 1" in _lib.lib().mc_last_error().decode()
        np.testing.assert_array_equal(s.read_frames(2, 1)[0], frames[2])


def test_tiff_size_mismatch_rejected(tmp_path):
    q = str(tmp_path / "b.tif")
    frames = [rng_frames(8, (1, 8, 8), np.uint8, 256)[0], rng_frames(8, (1, 9, 8), np.uint8, 256)[0]]
    ims = [PIL.fromarray(f) for f in frames]
    ims[0].save(q, save_all=True, append_images=ims[1:])
    with pytest.raises(_lib.McError, match="differs from the first directory"):
        api.Stack(q)


def _mrc_with_symdata(path, frames, mode, nsymbt):
    mrc.write_stack(str(path), frames, mode)
    b = bytearray(open(path, "rb").read())
    b[92:96] = struct.pack("<i", nsymbt)
    open(path, "wb").write(bytes(b[:1024]) + b"\x5a" * nsymbt + bytes(b[1024:]))


@pytest.mark.parametrize("mode,dtype", [(0, np.int8), (1, np.int16), (2, np.float32), (6, np.uint16),
                                        (12, np.float16)])
def test_mrc_and_mrcgz(tmp_path, mode, dtype):
    """Every pixel mode a plan decodes; 12 is MRC2014's IEEE half (including
    subnormals, infinities and a NaN), widened exactly on the host."""
    rng = np.random.default_rng(9 + mode)
    frames = (rng.normal(0, 50, (5, 33, 47)) if mode in (2, 12) else
              rng.integers(np.iinfo(dtype).min, np.iinfo(dtype).max, (5, 33, 47))).astype(dtype)
    p = tmp_path / "s.mrc"
    _mrc_with_symdata(p, frames, mode, 80)
    gz = tmp_path / "s.mrc.gz"
    gz.write_bytes(gzip.compress(p.read_bytes()))
    for path, fmt in [(p, "mrc"), (gz, "mrc-gz")]:
        with api.Stack(str(path)) as s:
            assert s.info["format_name"] == fmt and s.mode == mode and s.info["file_mode"] == mode
            np.testing.assert_array_equal(s.read_frames(), frames)
            np.testing.assert_array_equal(s.read_frames(3, 2), frames[3:5])
            np.testing.assert_array_equal(s.read_frames(1, 1), frames[1:2])  # backward seek
            np.testing.assert_array_equal(s.read_frame_float(4), frames[4].astype(np.float32))


def test_half_decode_special_values(tmp_path):
    h = np.arange(65536, dtype=np.uint32).astype(np.uint16).view(np.float16).reshape(1, 256, 256)
    p = tmp_path / "h.mrc"
    _mrc_with_symdata(p, h, 12, 0)
    with api.Stack(str(p)) as s:
        got = s.read_frame_float(0)
    want = h[0].astype(np.float32)
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(got), nan)
    np.testing.assert_array_equal(got[~nan], want[~nan])


def test_detection_order_and_rejects(tmp_path):
    frames = rng_frames(10, (2, 8, 8), np.uint8, 128).astype(np.int8)
    # no stamp: MRC only by a file name containing "mrc" (isMRC, func.cpp:557-578)
    a = tmp_path / "plain.mrc"
    mrc.write_stack(str(a), frames, 0)
    raw = bytearray(a.read_bytes())
    raw[208:212] = b"\0\0\0\0"
    a.write_bytes(bytes(raw))
    with api.Stack(str(a)) as s:
        assert s.info["format_name"] == "mrc"
    b = tmp_path / "plain.dat"
    b.write_bytes(a.read_bytes())
    with pytest.raises(_lib.McError, match="Only MRC, MRC-gz, TIFF"):
        api.Stack(str(b))
    # gzip without the stamp is not MRC-gz (isMRCZ, func.cpp:580-606)
    c = tmp_path / "nostamp.gz"
    c.write_bytes(gzip.compress(a.read_bytes()))
    with pytest.raises(_lib.McError, match="Only MRC, MRC-gz, TIFF"):
        api.Stack(str(c))
    with pytest.raises(_lib.McError):
        api.Stack(str(tmp_path / "missing.mrc"))
    t = tmp_path / "x.tif"
    write_tiff(str(t), rng_frames(11, (2, 8, 8), np.uint8, 256))
    with api.Stack(str(t)) as s:
        with pytest.raises(_lib.McError) as ei:
            s.read_frames(1, 2)
        assert ei.value.code == -1


def test_codec_edge_streams(tmp_path):
    """PackBits no-op byte (-128) and runs; an LZW stream that stops early."""
    frames = np.array([[[7] * 16 + list(range(16))]], dtype=np.uint8).reshape(1, 1, 32)
    p = tmp_path / "pb.tif"
    # hand-made PackBits strip: no-op, run of 16 sevens, literal 0..15
    strip = bytes([0x80, (1 - 16) & 0xff, 7, 15]) + bytes(range(16))
    write_tiff(str(p), frames, compression=32773)
    raw = bytearray(p.read_bytes())
    # replace the uncompressed strip (at offset 8, 32 bytes) with the PackBits one padded to 32 bytes
    raw[8:8 + 32] = strip.ljust(32, b"\x80")
    p.write_bytes(bytes(raw))
    with api.Stack(str(p)) as s:
        np.testing.assert_array_equal(s.read_frames()[0], frames[0])


@pytest.mark.parametrize("mode", [0, 1, 2, 6])
def test_mrcgz_matches_reference_reader(mode):
    """Golden decodes of the reference's own MRC-gz reader (MRCZ on MRC,
    mrcz.cpp + mrc.cpp compiled from the reference tree, read2DIm_32bit with
    gzseek; tests/golden/make_golden.py): mc_stack_read_frame_float gives the
    same floats bit for bit, including after a backward seek."""
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with api.Stack(os.path.join(here, f"stack_mode{mode}.mrc.gz")) as s:
        assert s.info["format_name"] == "mrc-gz" and s.mode == mode
        for k in (2, 0, 1):
            want = np.fromfile(os.path.join(here, f"ref_gz_decode_mode{mode}_f{k}.f32"), dtype=np.float32)
            got = s.read_frame_float(k).ravel()
            assert got.tobytes() == want.tobytes()
