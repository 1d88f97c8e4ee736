"""MRC I/O and frame decode pinned against the reference's own mrc.cpp.

The golden files in tests/golden/ were produced by the reference's MRC class
(tests/golden/make_golden.py over oracle/_ref/ref_mrc); when the reference
tree is present the harness is also run live.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from motioncorr1exp_b200 import mrc
from oracle import mc_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
ROOT = os.path.dirname(HERE)
REF = os.path.join(ROOT, "oracle", "_ref", "ref_mrc")


def _image():
    x = np.arange(17 * 13 * 2, dtype=np.float64).reshape(2, 13, 17)
    return (np.sin(x * 0.37) * 1000.0 + x * 0.125).astype(np.float32)


def test_header_layout():
    assert mrc.HEADER_DTYPE.itemsize == 1024
    assert mrc.HEADER_DTYPE.fields["map"][1] == 208
    assert mrc.HEADER_DTYPE.fields["nsymbt"][1] == 92
    assert mrc.HEADER_DTYPE.fields["label"][1] == 224


def test_writer_matches_reference_createMRC(tmp_path):
    ours = tmp_path / "ours.mrc"
    mrc.write_image(str(ours), _image())
    ref = open(os.path.join(GOLD, "ref_createMRC_17x13x2.mrc"), "rb").read()
    assert open(ours, "rb").read() == ref


@pytest.mark.parametrize("mode", [0, 1, 2, 6])
def test_decode_matches_reference_read2DIm_32bit(mode):
    frames, h = mrc.read_stack(os.path.join(GOLD, f"stack_mode{mode}.mrc"))
    assert int(h["mode"]) == mode
    for k in range(frames.shape[0]):
        ref = np.fromfile(os.path.join(GOLD, f"ref_decode_mode{mode}_f{k}.f32"), dtype=np.float32)
        got = O.decode_frame(frames[k].ravel(), mode).astype(np.float32)
        np.testing.assert_array_equal(got, ref)


def test_mode0_is_signed_char():
    frames, _ = mrc.read_stack(os.path.join(GOLD, "stack_mode0.mrc"))
    ref = np.fromfile(os.path.join(GOLD, "ref_decode_mode0_f0.f32"), dtype=np.float32)
    assert ref.min() < 0          # bytes >= 128 decode negative in the reference


def test_truncated_stack_is_rejected(tmp_path):
    p = tmp_path / "short.mrc"
    src = open(os.path.join(GOLD, "stack_mode2.mrc"), "rb").read()
    open(p, "wb").write(src[:-10])
    with pytest.raises(ValueError):
        mrc.read_stack(str(p))
    open(p, "wb").write(src[:500])
    with pytest.raises(ValueError):
        mrc.read_header(str(p))


def _reference_tree_present():
    r = subprocess.run(["bash", os.path.join(ROOT, "oracle", "build_ref.sh"), "--where"], capture_output=True)
    return r.returncode == 0


@pytest.mark.skipif(not _reference_tree_present(), reason="reference tree absent")
def test_live_reference_roundtrip(tmp_path):
    subprocess.run(["bash", os.path.join(ROOT, "oracle", "build_ref.sh")], check=True, capture_output=True)
    img = np.random.default_rng(0).normal(3, 2, (1, 31, 29)).astype(np.float32)
    raw = tmp_path / "in.f32"
    img.tofile(raw)
    ref = tmp_path / "ref.mrc"
    subprocess.run([REF, "write", str(ref), "29", "31", "1", str(raw)], check=True)
    ours = tmp_path / "ours.mrc"
    mrc.write_image(str(ours), img[0])
    assert open(ref, "rb").read() == open(ours, "rb").read()
    out = subprocess.run([REF, "header", str(ours)], check=True, capture_output=True, text=True).stdout.split()
    assert out[:4] == ["29", "31", "1", "2"]
