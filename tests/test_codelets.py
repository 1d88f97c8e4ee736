"""The generated FFT code (CPU only): the committed headers are what
motioncorr1exp_b200/csrc/gen_dft.py emits, and the prime-factor
(Good-Thomas) codelets' index maps -- Ruritanian input map, small DFTs
along each coprime factor with no twiddles, CRT output map -- give the DFT
(numpy's, forward and inverse) for every codelet length that has them."""
import importlib.util
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "motioncorr1exp_b200", "csrc")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_dft", os.path.join(CSRC, "gen_dft.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("which,fname", [("dft", "dft_gen.cuh"), ("codelets", "codelets_gen.cuh")])
def test_generated_headers_are_current(which, fname):
    out = subprocess.run([sys.executable, os.path.join(CSRC, "gen_dft.py"), which], capture_output=True,
                         text=True, check=True).stdout
    assert out == open(os.path.join(CSRC, fname)).read()


def test_prime_factor_maps_give_the_dft():
    G = _gen()
    lengths = [q for q in G.CODELETS if G.pfa_plan(q)]
    assert 70 in lengths and 35 in lengths and 60 in lengths
    for q in lengths:
        groups, ins, outs = G.pfa_indices(q)
        assert sorted(ins) == list(range(q)) and sorted(outs) == list(range(q))
        rng = np.random.default_rng(q)
        a = rng.normal(size=q) + 1j * rng.normal(size=q)
        strides = [1]
        for g in groups[:-1]:
            strides.append(strides[-1] * g)
        for inv in (False, True):
            b = a[ins].copy()
            for d, g in enumerate(groups):
                for base in range(q):
                    if (base // strides[d]) % g:
                        continue
                    idx = [base + r * strides[d] for r in range(g)]
                    b[idx] = np.fft.ifft(b[idx]) * g if inv else np.fft.fft(b[idx])
            got = np.empty(q, complex)
            got[outs] = b
            ref = np.fft.ifft(a) * q if inv else np.fft.fft(a)
            np.testing.assert_allclose(got, ref, atol=1e-9 * q)
