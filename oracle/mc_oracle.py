"""FP64 CPU oracle of the MotionCorr-1 frame-drift correction hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: it may be imported by
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference arm of
``bench.py``.  The product path (``motioncorr1exp_b200``) never imports it.

It restates, step by step and in float64 numpy, what ``dosefgpu_driftcorr``
(src-1125 of gepeng1983/motioncorr1exp) computes between reading the frames
and writing the corrected sum.  Every function cites the reference lines it
follows.  Index conventions, argmax tie-breaks, clamping rules and the
1/32-pixel quantisation of the sub-pixel search are kept exactly; only the
arithmetic is widened to FP64.

Parity status: the reference publishes no tests, fixtures or golden
vectors, and its build needs FFTW3, SP++ 3.0 and libtiff, none of which is
installed.  ``oracle/build_ref.sh`` compiles the reference's own sources
with project stand-ins for those (``oracle/stubs/``), and this oracle is
pinned against what they produce: the MRC and MRC-gz decode/encode
(``mrc.cpp``, ``mrcz.cpp``), ``func.cpp``'s crop size, crop, sub-pixel cosine
mask and display contrast/layout, the drift solve (``mfunc.h`` and the
least-squares steps of ``DFAlign.cu:875-948``; golden fixtures in
tests/golden/), and on the GPU the reference's forward spectra, pair stage
and shift-and-sum (``cufunc.cu`` with cuFFT, tests/test_gpu_reference_pair.py)
and its whole program, realignment iterations included
(tests/test_gpu_reference_full.py).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

try:  # multi-threaded pocketfft when available
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


SUBBOX = 16          # cufunc.cu:428
UPSCALE = 32         # cufunc.cu:441


# ---------------------------------------------------------------------------
# parameters
# ---------------------------------------------------------------------------
@dataclass
class Params:
    """Mirror of APARA (DFAlign.h:16-63) with the defaults of getDefaultPara
    (dosefgpu_driftcorr.cpp:8-58) plus the iteration fields of CDFAlign
    (DFAlign.h:75-76, defaults DFAlign.cu:15-16)."""
    crop_offsetx: int = 0
    crop_offsety: int = 0
    crop_nsam: int = 0
    bin: float = 1.0
    nStart: int = 0
    nEnd: int = 0
    nStartSum: int = 0
    nEndSum: int = 0
    bfactor: float = 150.0
    CCPeakSearchDim: int = 96
    FrameDistOffset: int = 2
    NoisePeakSize: int = 0
    kiThresh: float = 1.0
    bAlignToMid: int = 1
    iter: int = 0
    iterthres: float = 0.0


def verify_para(p: Params, nframe_file: int) -> Params:
    """Frame-range repair of VerifyPara (dosefgpu_driftcorr.cpp:60-103)."""
    p = Params(**p.__dict__)
    if p.nStart < 0:
        p.nStart = 0
    if p.nEnd >= nframe_file:
        p.nEnd = nframe_file - 1
    if p.nEnd <= p.nStart:
        p.nEnd = nframe_file - 1
    if p.nStartSum < p.nStart:
        p.nStartSum = p.nStart
    if p.nEndSum > p.nEnd:
        p.nEndSum = p.nEnd
    if p.nEndSum <= p.nStartSum:
        p.nEndSum = p.nEnd
    return p


def verify_crop_size(nx: int, ny: int, offx: int, offy: int, nsamout: int,
                     future_bin: float) -> int:
    """verifyCropSize (func.cpp:80-103): square crop side, even (x4 at bin 2)."""
    fb = float(np.float32(future_bin))
    if offx < 0 or offx >= nx or offy < 0 or offy >= ny or fb <= 0:
        return 0
    if nsamout <= 0:
        nsamout = min(nx - offx, ny - offy)
    if nx - offx < nsamout:
        nsamout = nx - offx
    if ny - offy < nsamout:
        nsamout = ny - offy
    if abs(fb - 1.0) < 0.0001:
        nsamout = nsamout // 2 * 2
    elif abs(fb - 2.0) < 0.0001:
        nsamout = nsamout // 4 * 4
    else:
        nsamout = nsamout // 2 * 2
    return nsamout


def binned_size(nsam_unbin: int, bin_: float) -> int:
    """nsam=(int)((float)nsamUnbin/bin)/2*2 (DFAlign.cu:515), float32 divide."""
    q = np.float32(nsam_unbin) / np.float32(bin_)
    return int(q) // 2 * 2


def pair_distance(nframe: int, fod: int) -> int:
    """dist of OD_GetNRow_All / OD_SetEquation_All (mfunc.h:52-54, 71-73)."""
    dist = nframe // 2 - fod
    if dist <= 0:
        dist = 1
    if dist > nframe // 2:
        dist = nframe // 2
    return dist


def pair_list(nframe: int, fod: int) -> list[tuple[int, int]]:
    """Pairs (i, j>=i+dist) in i-major, j-ascending order (mfunc.h:64-84)."""
    d = pair_distance(nframe, fod)
    return [(i, j) for i in range(nframe) for j in range(i + d, nframe)]


def design_matrix(pairs, nframe: int) -> np.ndarray:
    """Row r has ones on frame steps k in [i, j) (mfunc.h:79)."""
    A = np.zeros((len(pairs), nframe - 1))
    for r, (i, j) in enumerate(pairs):
        A[r, i:j] = 1.0
    return A


# ---------------------------------------------------------------------------
# frames
# ---------------------------------------------------------------------------
_MODE_DTYPE = {0: np.int8, 1: np.int16, 2: np.float32, 6: np.uint16, 100: np.uint8, 12: np.float16}


def decode_frame(raw: np.ndarray, mode: int) -> np.ndarray:
    """MRC::read2DIm_32bit (mrc.cpp:325-382): mode 0 is *signed* char; mode
    100 is the unsigned byte of an 8-bit TIFF strip (MRCT::read2DIm,
    mrct.cpp:137-150); mode 12 (MRC2014 IEEE half, no reference counterpart)
    widens exactly."""
    dt = _MODE_DTYPE.get(mode, np.float32)
    return np.asarray(raw).view(dt).astype(np.float64)


def stretch_image(img: np.ndarray, xscale: float = 1.0, yscale: float = 1.0) -> np.ndarray:
    """Image stretch of -scx/-scy (DFAlign.cu:503-504, 751-765): with
    r = float(1/yscale), c = float(1/xscale), pixel (y, x), y, x >= 1, takes
    the value at (int(float(y*r) + 0.5), int(float(x*c) + 0.5)); row 0 and
    column 0 are kept.  In place from the last pixel backwards in the
    reference, which reads only pixels not yet overwritten, so it equals a
    gather from the unstretched image."""
    xs = np.float32(1.0 / np.float64(np.float32(xscale)))
    ys = np.float32(1.0 / np.float64(np.float32(yscale)))
    if not (xs < 1.0 or ys < 1.0):
        return img
    ny, nx = img.shape
    rm = ((np.arange(ny, dtype=np.float32) * ys).astype(np.float64) + 0.5).astype(np.int64)
    cm = ((np.arange(nx, dtype=np.float32) * xs).astype(np.float64) + 0.5).astype(np.int64)
    out = np.array(img, copy=True)
    out[1:, 1:] = img[np.ix_(rm[1:], cm[1:])]
    return out


def apply_refs(raw: np.ndarray, dark=None, dark2=None, norm=None, norm2=None):
    """Two-reference dark/gain correction of DFAlign.cu:614-750.

    Returns (a, b): ``a`` feeds hbuf (first member of each pair, iterative
    sum and final sum), ``b`` feeds hbuf2 (second member of each pair).
    A single-frame reference means dark2 = 0 / norm2 = 1 (DFAlign.cu:648-651,
    688-691).  Without references b == a (DFAlign.cu:749).
    """
    raw = np.asarray(raw, dtype=np.float64)
    if dark is not None and dark2 is None:
        dark2 = np.zeros_like(raw)
    if norm is not None and norm2 is None:
        norm2 = np.ones_like(raw)
    if norm is not None and dark is not None:
        return (raw - dark) * norm, (raw - dark2) * norm2
    if norm is not None:
        return raw * norm, raw * norm2
    if dark is not None:
        return raw - dark, raw - dark2
    return raw, raw


def forward_spectrum(img: np.ndarray, offx: int, offy: int, nu: int, n: int) -> np.ndarray:
    """crop2fft (func.cpp:157-173) + cufftExecR2C (cufunc.cu:223-227) +
    Fourier-crop GPUMemBinD2D (cufunc.cu:162-176).

    Returns the un-normalised half spectrum, shape (n, n//2+1), row = ky
    (ky >= n/2 meaning ky-n), column = kx -- the reference's device layout.
    Binning keeps rows [0, n/2) and [nu-n/2, nu) with no rescale.
    """
    crop = np.asarray(img, dtype=np.float64)[offy:offy + nu, offx:offx + nu]
    F = _rfft2(crop)
    if nu == n:
        return F
    h = n // 2
    out = np.empty((n, h + 1), dtype=np.complex128)
    out[:h] = F[:h, :h + 1]
    out[h:] = F[nu - h:, :h + 1]
    return out


def bfactor_mask(n: int, bfactor: float) -> np.ndarray:
    """MkPosList(MASK*) (cufunc.cu:309-341): z = (-1)^(x+y) exp(m r^2),
    m = -0.5*bfactor/n/n rounded to float (cufunc.cu:316)."""
    m = float(np.float32(-0.5 * float(np.float32(bfactor)) / n / n))
    ky = np.arange(n)
    y = np.where(ky < n // 2, ky, ky - n)[:, None]
    x = np.arange(n // 2 + 1)[None, :]
    r2 = x * x + y * y
    sign = np.where((x + y) % 2 == 0, 1.0, -1.0)
    return sign * np.exp(m * r2)


def cc_map(Fa: np.ndarray, Fb: np.ndarray, mask: np.ndarray, n: int) -> np.ndarray:
    """cuShiftCC with zero shift (cufunc.cu:343-370) followed by the
    un-normalised C2R (cufunc.cu:229-233): C = Fa conj(Fb) z / ((n/2+1) n)."""
    size = (n // 2 + 1) * n
    C = Fa * np.conj(Fb) * (mask / size)
    return _irfft2(C, s=(n, n)) * float(n * n)


def cc_box(ccmap: np.ndarray, n: int, box: int) -> np.ndarray:
    """The pbx x pbx window FindShift copies out (cufunc.cu:398-407)."""
    ori = (n - box) // 2
    return ccmap[ori:ori + box, ori:ori + box].copy()


def cosmask16_weights() -> np.ndarray:
    """cosmask2d (func.cpp:348-370) on the 16x16 half spectrum, shape (16, 9)."""
    n = SUBBOX
    h = n // 2
    w = np.zeros((n, h + 1))
    step = math.pi / h
    for j in range(n):
        ky = j if j < h else j - n
        for i in range(h + 1):
            r = int(math.sqrt(float(i * i + ky * ky)))
            w[j, i] = math.cos(r * step) / 2 + 0.5 if r < h else 0.0
    return w


_W16 = None


def integer_peak(box_map: np.ndarray, nps: int) -> tuple[int, int]:
    """Integer argmax of FindShift (cufunc.cu:409-424): y outer, x inner,
    strict '>' starting from -1e9, optional centre exclusion (wNoise=nps-1)."""
    box = box_map.shape[0]
    wnoise = nps - 1
    vals = np.asarray(box_map, dtype=np.float64).copy()
    jj, ii = np.mgrid[0:box, 0:box]
    excl = (np.abs(ii - box // 2) <= wnoise) & (np.abs(jj - box // 2) <= wnoise)
    vals[excl] = -np.inf
    flat = vals.ravel()
    k = int(np.argmax(flat))          # first occurrence of the maximum
    if not flat[k] > -1e9:
        return 0, 0
    return k % box, k // box


def upsampled_subbox(box_map: np.ndarray, offx: int, offy: int) -> np.ndarray:
    """16x16 sub-box -> R2C -> cosmask2d -> zero-pad to 512 -> C2R
    (cufunc.cu:437-455, func.cpp:10-24), un-normalised like FFTW."""
    global _W16
    if _W16 is None:
        _W16 = cosmask16_weights()
    sub = np.asarray(box_map, dtype=np.float64)[offy:offy + SUBBOX, offx:offx + SUBBOX]
    S = np.fft.rfft2(sub) * _W16
    pad = SUBBOX * UPSCALE
    P = np.zeros((pad, pad // 2 + 1), dtype=np.complex128)
    h = SUBBOX // 2
    P[:h, :h + 1] = S[:h]
    P[pad - h:, :h + 1] = S[h:]
    return np.fft.irfft2(P, s=(pad, pad)) * float(pad * pad)


def find_shift(box_map: np.ndarray, n: int, nps: int = 0):
    """FindShift (cufunc.cu:396-497).

    Returns (sx, sy, cc, ix, iy): the shift in 1/32-px units (as floats),
    the CC value max/n/n/256, and the integer box peak (ix, iy).
    """
    box = box_map.shape[0]
    wnoise = nps - 1
    ix, iy = integer_peak(box_map, nps)
    offx = ix - SUBBOX // 2
    offy = iy - SUBBOX // 2
    if offx + SUBBOX > box:
        offx = box - SUBBOX
    elif offx < 0:
        offx = 0
    if offy + SUBBOX > box:
        offy = box - SUBBOX
    elif offy < 0:
        offy = 0
    f = upsampled_subbox(box_map, offx, offy)
    pad = SUBBOX * UPSCALE
    ox = (box // 2 - offx) * UPSCALE
    oy = (box // 2 - offy) * UPSCALE
    wns = UPSCALE * wnoise
    vals = f.copy()
    jj, ii = np.mgrid[0:pad, 0:pad]
    excl = (np.abs(ii - ox) <= wns) & (np.abs(jj - oy) <= wns)
    vals[excl] = -np.inf
    flat = vals.ravel()
    k = int(np.argmax(flat))
    best0 = f[0, 0]
    if flat[k] > best0:
        sxp, syp, best = k % pad, k // pad, flat[k]
    else:
        sxp, syp, best = 0, 0, best0
    sx = offx + sxp / float(UPSCALE) - box // 2
    sy = offy + syp / float(UPSCALE) - box // 2
    cc = best / n / n / SUBBOX / SUBBOX
    return sx, sy, cc, ix, iy


# ---------------------------------------------------------------------------
# least squares + outlier rejection
# ---------------------------------------------------------------------------
def lsq(A: np.ndarray, b: np.ndarray) -> np.ndarray:
    """lsSolver(A, b) (DFAlign.cu:915): complex LS == two real LS with one A."""
    rhs = np.stack([b.real, b.imag], axis=1)
    sol, *_ = np.linalg.lstsq(A, rhs, rcond=None)
    return sol[:, 0] + 1j * sol[:, 1]


def od_threshold(A: np.ndarray, b: np.ndarray, ki: np.ndarray, kithresh: float):
    """OD_Threshold (mfunc.h:101-146) with Min_VectorIndex (mfunc.h:86-99).

    Rows ordered by ascending ki (first minimum wins ties); keep the prefix
    ending at the last position >= cols whose ki < kithresh (else the first
    cols rows); grow by one row until rank == cols; return the kept rows in
    ascending original order.
    """
    ncols = A.shape[1]
    order = list(np.argsort(ki, kind="stable"))
    thr = float(np.float32(kithresh))
    i = len(order) - 1
    while i >= ncols:
        if ki[order[i]] < thr:
            break
        i -= 1
    ii = i
    while True:
        good = sorted(order[:ii + 1])
        rank = np.linalg.matrix_rank(A[good]) if good else 0
        ii += 1
        if not (rank < ncols and ii < len(order)):
            break
    return good


# ---------------------------------------------------------------------------
# phase shift / sum
# ---------------------------------------------------------------------------
def phase_shift(F: np.ndarray, sx: float, sy: float) -> np.ndarray:
    """cuShift (cufunc.cu:372-393): F * exp(i 2pi (sx*kx + sy*ky)/n), ky signed."""
    n = F.shape[0]
    ky = np.arange(n)
    y = np.where(ky < n // 2, ky, ky - n)[:, None]
    x = np.arange(n // 2 + 1)[None, :]
    return F * np.exp(1j * (2.0 * math.pi / n) * (sx * x + sy * y))


def spectrum_to_image(Fsum: np.ndarray) -> np.ndarray:
    """C2R then x 1/nsam^2 (DFAlign.cu:1289-1292)."""
    n = Fsum.shape[0]
    return _irfft2(Fsum, s=(n, n))


def raw_sum_image(F: list, first: int, last: int) -> np.ndarray:
    """Unaligned sum of spectra first..last (run positions): the raw even/odd
    sums of DFAlign.cu:807-813 added at :821-824, transformed and scaled as
    the "-srs" output (:851-858)."""
    S = np.zeros_like(F[first])
    for k in range(first, last + 1):
        S = S + F[k]
    return spectrum_to_image(S)


# ---------------------------------------------------------------------------
# quick-look displays of -dsp 1 (DFAlign.cu:73-178, 841-849, 1270-1286)
# ---------------------------------------------------------------------------
DISPDIM = 400  # DFAlign.h:13


def hist_min_max(buf: np.ndarray, threshold: float = 0.005):
    """histMinMax (func.cpp:372-420): 400-bin histogram, the lowest and the
    highest `threshold` fraction cut off; float arithmetic."""
    b = np.asarray(buf, np.float32).ravel()
    mn, mx = np.float32(b.min()), np.float32(b.max())
    if mn >= mx:
        return mn, mx
    nbin = 400
    step = np.float32((mx - mn) / np.float32(nbin))
    ids = ((b - mn) / step).astype(np.int64)
    ids[ids >= nbin] = nbin - 1
    hist = np.bincount(ids, minlength=nbin)
    percent = int(b.size * threshold)
    c = np.cumsum(hist)
    i = int(np.argmax(c > percent))
    lo = np.float32(mn + np.float32(i) * step)
    c2 = np.cumsum(hist[::-1][:-1])              # bins nbin-1 down to 1
    hi = mx
    if np.any(c2 > percent):
        k = int(np.argmax(c2 > percent))         # bin nbin-1-k
        hi = np.float32(mx - np.float32(k) * step)
    return lo, hi


def display_short(buf: np.ndarray) -> np.ndarray:
    """buf2DispShort (func.cpp:440-455): linear map of [min, max] to 0..255."""
    b = np.asarray(buf, np.float32)
    mn, mx = hist_min_max(b)
    out = np.zeros(b.shape, np.int16)
    if mn >= mx:
        return out
    scale = np.float32(255.0) / np.float32(mx - mn)
    v = ((b - mn) * scale).astype(np.int16)
    out = np.where(b <= mn, 0, np.where(b >= mx, 255, v)).astype(np.int16)
    return out


def modulus_layout(L: np.ndarray) -> np.ndarray:
    """FFTModulusToDispBuf (func.cpp:459-489): a half-spectrum image L
    (n, n/2+1), rows ky, placed as the centred display buffer (n, n+2): the
    right half from L, the left half mirrored through the centre, row 0's
    left half repeating row 1's."""
    n = L.shape[0]
    h = n // 2
    out = np.zeros((n, n + 2), dtype=np.asarray(L).dtype)
    out[h:, h:n + 1] = L[:h, :]
    out[:h, h:n + 1] = L[h:, :]
    for j in range(1, n):
        out[j, :h] = out[n - j, n - np.arange(h)]
    out[0, :h] = out[1, :h]
    return out


def modulus_display(F: np.ndarray, scale: float = 1e-4) -> np.ndarray:
    """cuFFTLogModulus (cufunc.cu:178-188) + FFTModulusToDispBuf
    (func.cpp:459-489): log(1 + |F| scale) as the centred n x n image."""
    return modulus_layout(np.log1p(np.abs(F) * scale))[:, :F.shape[0]]


def bin_spectrum(F: np.ndarray, d: int = DISPDIM) -> np.ndarray:
    """GPUMemBinD2H (cufunc.cu:147-161): rows ky < d/2 and the last d/2 rows,
    kx <= d/2 of a half spectrum (rows ky)."""
    h = d // 2
    return np.concatenate([F[:h, :h + 1], F[F.shape[0] - h:, :h + 1]], axis=0)


def quicklook(F: np.ndarray, which: int) -> np.ndarray:
    """The three displays: 0 raw FFT and 2 corrected FFT from a sum spectrum
    (BinFFTDispBufToChar, func.cpp:524-556: R2C of the modulus image, Fourier
    bin to 400, C2R / 400^2), 1 the sum itself binned (ImageOutputThread,
    DFAlign.cu:73-93: C2R unnormalised)."""
    d = DISPDIM
    if which == 1:
        img = np.fft.irfft2(bin_spectrum(F, d), s=(d, d)) * (d * d)
    else:
        M = modulus_display(F)
        img = np.fft.irfft2(bin_spectrum(np.fft.rfft2(M), d), s=(d, d))
    return display_short(img)


def fsc_table(F: list, first: int, last: int, sum_shift, align_to_mid: bool, drift) -> np.ndarray:
    """PlotFSC (DFAlign.cu:212-326) in FP64 over spectra (n, n//2+1).

    Even/odd halves: run positions first, first+2, ... and first+1, ...
    (raw: DFAlign.cu:806-812; aligned: DFAlign.cu:1142-1179, 1237-1244, the
    first frame shifted only with -atm 1).  Shells: r = sqrtf(x^2+y^2) in
    float over the MkPosList coordinates (cufunc.cu:309-339), skipped when
    int(r) <= 0 or r >= n/2+1, shell int(r/step) with step = n/400; along the
    drift when float(|x dx + y dy| / r) > float(cos 45 deg) for the unit drift
    (x axis below 0.1 px).  Returns (nbox, 5): Nq%, D_Raw, U_Raw, D_Corr,
    U_Corr, each x/sqrt(aa*bb) or 0 when aa*bb <= 1e-5."""
    n = F[first].shape[0]
    step = n // 400
    nsamc = n // 2 + 1
    nbox = nsamc // step + 1
    raw = [np.zeros_like(F[first]), np.zeros_like(F[first])]
    cor = [np.zeros_like(F[first]), np.zeros_like(F[first])]
    for k in range(first, last + 1):
        h = (k - first) & 1
        raw[h] = raw[h] + F[k]
        apply = not (k == first and not align_to_mid)
        cor[h] = cor[h] + (phase_shift(F[k], sum_shift[k][0], sum_shift[k][1]) if apply else F[k])
    d = complex(drift[0], drift[1])
    d = d / abs(d) if abs(d) > 0.1 else complex(1.0, 0.0)
    ky = np.arange(n)
    y = np.where(ky < n // 2, ky, ky - n)[:, None].astype(np.int64)
    x = np.arange(nsamc)[None, :].astype(np.int64)
    r = np.sqrt((x * x + y * y).astype(np.float32))
    keep = (r.astype(np.int64) > 0) & (r < np.float32(nsamc))
    sid = (r / np.float32(step)).astype(np.int64)
    with np.errstate(divide="ignore", invalid="ignore"):  # r = 0 is outside `keep`
        ang = (np.abs(x * d.real + y * d.imag) / r.astype(np.float64)).astype(np.float32)
    along = ang > np.float32(math.cos(math.pi / 4))
    out = np.zeros((nbox, 5))
    out[:, 0] = np.arange(nbox) * 100.0 / nbox
    for col, (a, b) in ((1, raw), (3, cor)):
        prods = [(a * b.conj()).real, np.abs(a) ** 2, np.abs(b) ** 2]
        for j, cls in ((0, along), (1, ~along)):
            m = keep & cls
            s = [np.bincount(sid[m], weights=p[m], minlength=nbox) for p in prods]
            t = s[1] * s[2]
            out[:, col + j] = np.where(t > 1e-5, s[0] / np.sqrt(np.where(t > 0, t, 1.0)), 0.0)
    return out


def count_sum(frames: np.ndarray, mode: int, offx: int, offy: int, nu: int, first: int,
              last: int) -> np.ndarray:
    """Exact integer sum of the decoded raw pixels (read2DIm_32bit,
    mrc.cpp:325-382) of run positions first..last over the square crop (the
    count sums of the precision method; no reference counterpart)."""
    dt = _MODE_DTYPE[mode]
    acc = np.zeros((nu, nu), dtype=np.int64)
    for k in range(first, last + 1):
        acc += np.asarray(frames[k]).view(dt)[offy:offy + nu, offx:offx + nu].astype(np.int64)
    return acc


# ---------------------------------------------------------------------------
# frame-to-sum objective of the added gradient refinement (no reference
# counterpart: north-star method 3), FP64
# ---------------------------------------------------------------------------
def sum_objective(F: list, shifts: np.ndarray, bfactor: float):
    """J(s) = sum_w h(kx) w(kx,ky) |S|^2 with S = sum_k F_k exp(+i w.s_k),
    w the B-factor weight exp(-0.5*bft*r^2/n^2) and h the half-spectrum
    multiplicity (1 at kx = 0, n/2; 2 otherwise).  Returns (J, grad (F, 2),
    hess (F, 3) = (xx, xy, yy) diagonal 2x2 blocks) where, with
    P_k = F_k exp(i w.s_k) and u_k = conj(S - P_k) P_k,
        grad_k = -2 sum h w  w_vec Im(u_k),  hess_k = -2 sum h w w_vec w_vec^T Re(u_k).
    Each P_k is formed twice (once for S, once for its terms) so that only
    S and one P_k are held at a time.
    """
    n = F[0].shape[0]
    ky = np.arange(n)
    y = np.where(ky < n // 2, ky, ky - n)[:, None].astype(np.float64)
    x = np.arange(n // 2 + 1)[None, :].astype(np.float64)
    wgt = np.exp(-0.5 * float(bfactor) / n / n * (x * x + y * y))
    h = np.where((x == 0) | (x == n // 2), 1.0, 2.0)
    hw = h * wgt
    ox = 2.0 * math.pi * x / n
    oy = 2.0 * math.pi * y / n

    def term(k):
        return F[k] * np.exp(1j * (ox * shifts[k][0] + oy * shifts[k][1]))
    S = np.zeros_like(F[0], dtype=np.complex128)
    for k in range(len(F)):
        S += term(k)
    J = float(np.sum(hw * np.abs(S) ** 2))
    grad = np.zeros((len(F), 2))
    hess = np.zeros((len(F), 3))
    for k in range(len(F)):
        Pk = term(k)
        u = np.conj(S - Pk) * Pk
        grad[k, 0] = -2.0 * np.sum(hw * ox * u.imag)
        grad[k, 1] = -2.0 * np.sum(hw * oy * u.imag)
        hess[k, 0] = -2.0 * np.sum(hw * ox * ox * u.real)
        hess[k, 1] = -2.0 * np.sum(hw * ox * oy * u.real)
        hess[k, 2] = -2.0 * np.sum(hw * oy * oy * u.real)
    return J, grad, hess


def newton_steps(F: list, shifts: np.ndarray, bfactor: float) -> np.ndarray:
    """Per-frame block-Newton step -H_k^{-1} g_k of sum_objective at sum
    shifts ``shifts`` (F, 2): the update the gradient refinement would take
    from there in FP64 (zero for a frame whose block is not negative
    definite).  Its length bounds how far a refined solution is from a fixed
    point of the FP64 iteration."""
    _, g, hs = sum_objective(F, shifts, bfactor)
    out = np.zeros((len(F), 2))
    for k in range(len(F)):
        a, b, c = hs[k]
        det = a * c - b * b
        if a < 0.0 and det > 0.0:
            out[k, 0] = -(c * g[k, 0] - b * g[k, 1]) / det
            out[k, 1] = -(-b * g[k, 0] + a * g[k, 1]) / det
    return out


# ---------------------------------------------------------------------------
# whole movie
# ---------------------------------------------------------------------------
def corrected_sum(Fa: list, shift: np.ndarray, p: Params, nstart: int, nz_file: int,
                  want_image: bool = True):
    """The corrected sum of DFAlign.cu:1114-1292 from per-step shifts
    ``shift`` (nframe-1, complex): frames nStartSum..nEndSum, each shifted
    by -cumulative + mid (mid = the steps up to nz/2+1 with -atm 1,
    DFAlign.cu:1132-1139); the first summed frame is left unshifted unless
    -atm 1 (DFAlign.cu:1148).  Returns (sum_shift per frame, image or None)."""
    nframe = len(Fa)
    nss = p.nStartSum - nstart
    nes = p.nEndSum - nstart
    if nss <= 0:
        nss = 0
    if nes <= nss or nes >= nframe:
        nes = nframe - 1
    mid = 0.0 + 0.0j
    if p.bAlignToMid:
        ref = nz_file // 2 + 1
        if ref < nstart:
            ref = nstart
        # the reference reads past shift[] when ref-nstart > nframe-1; clamp
        for jj in range(min(ref - nstart, nframe - 1)):
            mid += shift[jj]
    total = 0.0 + 0.0j
    for jj in range(1, nss + 1):          # DFAlign.cu:1142-1146
        total += shift[jj - 1]
    sum_shift = np.zeros(nframe, dtype=np.complex128)
    S = None
    for k in range(nss, nes + 1):
        if k > nss:
            total += shift[k - 1]
        s = -total + mid
        sum_shift[k] = s
        if k == nss and not p.bAlignToMid:
            term = Fa[k]
        else:
            term = phase_shift(Fa[k], s.real, s.imag)
        S = term if S is None else S + term
    return sum_shift, (spectrum_to_image(S) if want_image else None)


@dataclass
class Result:
    nsam: int
    nsam_unbin: int
    pairs: list
    pair_shift: np.ndarray          # complex, per pair (1/32 px)
    pair_cc: np.ndarray
    pair_peak: np.ndarray           # (P, 2) integer box peak (x, y)
    ki1: np.ndarray                 # first-round residuals
    goodlist: list
    ki2: np.ndarray                 # second-round residuals
    shift: np.ndarray               # per-step shifts after iteration (complex)
    frame_shift: np.ndarray         # cumulative per-frame shifts (complex)
    sum_shift: np.ndarray           # shift applied to each summed frame
    image: Optional[np.ndarray]
    frame_mean: np.ndarray
    iter_log: list = field(default_factory=list)
    boxes: Optional[np.ndarray] = None  # (P, box, box) CC windows when asked for
    spectra: Optional[list] = None      # set-A spectra of the aligned frames when asked for


def align_movie(frames: np.ndarray, mode: int, p: Params, nz_file: Optional[int] = None,
                refs: Optional[dict] = None, want_image: bool = True, stretch=(1.0, 1.0),
                keep_boxes: bool = False, keep_spectra: bool = False) -> Result:
    """ThreadFunc_cuAlign (DFAlign.cu:456-1355) on decoded frames.

    ``frames``: raw stack (nz, ny, nx) in the file's pixel type.  ``p`` must
    already be repaired by verify_para (the CLI does it before RunAlign).
    ``keep_boxes`` keeps every pair's CC window (hboxmap, DFAlign.cu:880) for
    near-tie checks; ``keep_spectra`` the frames' spectra (hbuf).
    """
    nz, ny, nx = frames.shape
    if nz_file is None:
        nz_file = nz
    bin_ = float(np.float32(p.bin))
    nu = verify_crop_size(nx, ny, p.crop_offsetx, p.crop_offsety, p.crop_nsam, bin_)
    if nu <= 0:
        raise ValueError("Error: Wrong image Size.")
    n = binned_size(nu, bin_)
    nstart = max(p.nStart, 0)
    nend = min(p.nEnd, nz_file - 1)
    nframe = nend - nstart + 1
    refs = refs or {}
    mask = bfactor_mask(n, p.bfactor)
    box = p.CCPeakSearchDim

    # (B) ingest: DFAlign.cu:710-820
    Fa, Fb, fmean = [], [], []
    for f in range(nstart, nend + 1):
        raw = decode_frame(frames[f], mode)
        a, b = apply_refs(raw, refs.get("dark"), refs.get("dark2"), refs.get("norm"), refs.get("norm2"))
        if b is a:
            a = b = stretch_image(a, *stretch)
        else:
            a, b = stretch_image(a, *stretch), stretch_image(b, *stretch)
        sa = forward_spectrum(a, p.crop_offsetx, p.crop_offsety, nu, n)
        sb = sa if b is a else forward_spectrum(b, p.crop_offsetx, p.crop_offsety, nu, n)
        Fa.append(sa)
        Fb.append(sb)
        fmean.append(sa[0, 0].real / n / n)

    # (C) pairs: DFAlign.cu:875-905
    pairs = pair_list(nframe, p.FrameDistOffset)
    A = design_matrix(pairs, nframe)
    bvec = np.zeros(len(pairs), dtype=np.complex128)
    cc = np.zeros(len(pairs))
    peaks = np.zeros((len(pairs), 2), dtype=np.int64)
    boxes = np.zeros((len(pairs), box, box)) if keep_boxes else None
    for r, (i, j) in enumerate(pairs):
        bm = cc_box(cc_map(Fa[i], Fb[j], mask, n), n, box)
        if keep_boxes:
            boxes[r] = bm
        sx, sy, c, ix, iy = find_shift(bm, n, p.NoisePeakSize)
        bvec[r] = sx + 1j * sy
        cc[r] = c
        peaks[r] = (ix, iy)

    # (C) solve: DFAlign.cu:914-948
    shift = lsq(A, bvec)
    ki1 = np.abs(A @ shift - bvec)
    good = od_threshold(A, bvec, ki1, p.kiThresh)
    A2, b2 = A[good], bvec[good]
    shift = lsq(A2, b2)
    ki2 = np.abs(A2 @ shift - b2)

    # (D) iterative realignment: DFAlign.cu:950-1071
    newshift = np.concatenate([[0.0 + 0.0j], np.cumsum(shift)])
    oldshift = newshift.copy()
    rmsd = 0.0
    iter_log = []
    j = 0
    converged = False
    ith = float(np.float32(p.iterthres))
    while j < p.iter and not converged:
        S = np.zeros_like(Fa[0])
        for k in range(nframe):
            S = S + phase_shift(Fa[k], -oldshift[k].real, -oldshift[k].imag)
        ns = np.zeros(nframe, dtype=np.complex128)
        ccs = np.zeros(nframe)
        for k in range(nframe):
            bm = cc_box(cc_map(S, Fa[k], mask, n), n, box)
            sx, sy, c, _, _ = find_shift(bm, n, p.NoisePeakSize)
            ns[k] = sx + 1j * sy
            ccs[k] = c
        newshift = ns
        refshift = newshift[0]
        diff = oldshift - newshift
        oldshift = newshift - refshift
        rmsd += float(np.sum(diff.real ** 2 + diff.imag ** 2))
        rmsd /= nframe
        if rmsd < ith * ith:
            converged = True
        iter_log.append({"newshift": ns.copy(), "cc": ccs, "rmsd": rmsd, "converged": converged})
        j += 1
    # DFAlign.cu:1061-1071 converts back unconditionally (also when itr=0)
    shift = oldshift[1:] - oldshift[:-1]

    frame_shift = np.concatenate([[0.0 + 0.0j], np.cumsum(shift)])

    # (E) final sum: DFAlign.cu:1114-1292
    sum_shift, image = corrected_sum(Fa, shift, p, nstart, nz_file, want_image)
    return Result(nsam=n, nsam_unbin=nu, pairs=pairs, pair_shift=bvec, pair_cc=cc,
                  pair_peak=peaks, ki1=ki1, goodlist=good, ki2=ki2, shift=shift,
                  frame_shift=frame_shift, sum_shift=sum_shift, image=image,
                  frame_mean=np.array(fmean), iter_log=iter_log, boxes=boxes,
                  spectra=Fa if keep_spectra else None)
