"""Python mirror of the reference's alignment interface over libmc.

``Params`` carries the APARA fields (DFAlign.h:16-63) under the reference's
names; ``Plan`` wraps one mc_plan (one stack geometry on one GPU) and exposes
the stages of CDFAlign::ThreadFunc_cuAlign (DFAlign.cu:456-1355).  Every
call goes through the C ABI of libmc.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, fields
from typing import Callable, Optional

import numpy as np

from . import _lib as L


@dataclass
class Params:
    """APARA with the defaults of getDefaultPara (dosefgpu_driftcorr.cpp:8-58)."""
    crop_offsetx: int = 0
    crop_offsety: int = 0
    crop_nsam: int = 0
    bin: float = 1.0
    nStart: int = 0
    nEnd: int = 0
    nStartSum: int = 0
    nEndSum: int = 0
    GPUNum: int = 0
    bfactor: float = 150.0
    CCPeakSearchDim: int = 96
    FrameDistOffset: int = 2
    NoisePeakSize: int = 0
    kiThresh: float = 1.0
    bAlignToMid: int = 1
    iter: int = 0
    iterthres: float = 0.0
    refine: int = 0

    def to_c(self) -> L.McParams:
        c = L.McParams()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c

    @classmethod
    def from_c(cls, c: L.McParams) -> "Params":
        return cls(**{f.name: getattr(c, f.name) for f in fields(cls)})


def default_params() -> Params:
    c = L.McParams()
    L.lib().mc_default_params(C.byref(c))
    return Params.from_c(c)


def verify_params(p: Params, nz: int) -> Params:
    """VerifyPara (dosefgpu_driftcorr.cpp:60-118); raises McError on abort."""
    c = p.to_c()
    L.check(L.lib().mc_verify_params(C.byref(c), nz))
    return Params.from_c(c)


MODE_U8 = 100  # unsigned 8-bit pixels (8-bit TIFF)
MODE_F16 = 12  # IEEE half floats (MRC2014 mode 12): frames held in half the bytes of mode 2
_WORD_LENGTH = {0: 1, 1: 2, 2: 4, 6: 2, MODE_U8: 1, MODE_F16: 2}
KERNEL_KINDS = 9


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


_schedules_loaded = False


def _load_schedules() -> None:
    """Installs the autotuner's cached pair-stage schedules once per process
    (MC_SCHEDULES=0 keeps the built-in choices)."""
    global _schedules_loaded
    if _schedules_loaded:
        return
    _schedules_loaded = True
    if os.environ.get("MC_SCHEDULES", "1") == "0":
        return
    from . import autotune
    autotune.load()


class Plan:
    """One stack geometry on one GPU (mc_plan_create)."""

    def __init__(self, params: Params, nx: int, ny: int, nz: int, mode: int,
                 log: Optional[Callable[[str], None]] = None, cap_frames: int = 0, cap_pairs: int = 0,
                 spectrum_slots: Optional[int] = None):
        """spectrum_slots: None or 0 keeps every frame's spectrum in HBM when
        it fits (else as many as fit); n >= 4 holds at most n spectra and
        recomputes the others' forward transforms when a stage needs them
        (mc_plan_create_slots)."""
        self._lib = L.lib()
        _load_schedules()
        h = C.c_void_p()
        c = params.to_c()
        if spectrum_slots:
            L.check(self._lib.mc_plan_create_slots(C.byref(c), nx, ny, nz, mode, cap_frames, cap_pairs,
                                                   spectrum_slots, C.byref(h)))
        elif cap_frames or cap_pairs:
            L.check(self._lib.mc_plan_create_capacity(C.byref(c), nx, ny, nz, mode, cap_frames, cap_pairs,
                                                      C.byref(h)))
        else:
            L.check(self._lib.mc_plan_create(C.byref(c), nx, ny, nz, mode, C.byref(h)))
        self._h = h
        self.params = params
        self._logcb = None
        if log is not None:
            self.set_log(log)
        self._refresh_info()

    def _refresh_info(self) -> None:
        info = L.McInfo()
        L.check(self._lib.mc_plan_info(self._h, C.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in L.McInfo._fields_}

    def reframe(self, params: Params, nz: int) -> None:
        """New frame range / pair distance / threshold on the same geometry
        (mc_plan_reframe); frames must be loaded or bound again."""
        c = params.to_c()
        L.check(self._lib.mc_plan_reframe(self._h, C.byref(c), nz))
        self.params = params
        self._refresh_info()

    def bind_frames_device(self, dev_ptr: int) -> None:
        """Read the run's frames in place from device memory (0 unbinds)."""
        L.check(self._lib.mc_plan_bind_frames_device(self._h, C.c_void_p(dev_ptr) if dev_ptr else None))

    # -- lifecycle
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mc_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def stream(self) -> int:
        return int(self._lib.mc_plan_stream(self._h) or 0)

    @property
    def nsam(self) -> int:
        return self.info["nsam"]

    @property
    def nframe(self) -> int:
        return self.info["nframe"]

    @property
    def npairs(self) -> int:
        return self.info["npairs"]

    @property
    def spectrum_slots(self) -> int:
        """0 when every frame's spectrum stays in HBM, else the spectra held."""
        return self.info["spectrum_slots"]

    @property
    def forward_recomputes(self) -> int:
        """Forward transforms run again for spectra the plan had given up."""
        self._refresh_info()
        return self.info["forward_recomputes"]

    def set_log(self, fn: Callable[[str], None]) -> None:
        def _cb(text, _user):
            fn(text.decode(errors="replace"))
        self._logcb = L.LOG_FN(_cb)
        self._lib.mc_plan_set_log(self._h, self._logcb, None)

    # -- inputs
    def set_refs(self, dark=None, dark2=None, norm=None, norm2=None) -> None:
        keep = []

        def p(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32)
            keep.append(a)
            return _ptr(a)
        L.check(self._lib.mc_plan_set_refs(self._h, p(dark), p(dark2), p(norm), p(norm2)))
        self.info["two_sets"] = int(dark is not None or norm is not None)

    def set_stretch(self, xscale: float = 1.0, yscale: float = 1.0) -> None:
        """-scx/-scy: nearest-neighbour magnification correction (factors >= 1)."""
        L.check(self._lib.mc_plan_set_stretch(self._h, xscale, yscale))

    def load_frames(self, frames: np.ndarray, first: int = 0) -> None:
        """Raw frames (count, ny, nx) in the plan's MRC pixel type, host memory."""
        a = np.ascontiguousarray(frames)
        if a.dtype.itemsize != _WORD_LENGTH[self.info["mode"]]:
            raise ValueError(f"frames of {a.dtype} do not match MRC mode {self.info['mode']}")
        count = a.shape[0] if a.ndim == 3 else 1
        L.check(self._lib.mc_plan_load_frames(self._h, _ptr(a), first, count))
        self._lib_keep = a  # the copy is asynchronous on the plan stream

    def load_frames_device(self, dev_ptr: int, first: int, count: int) -> None:
        L.check(self._lib.mc_plan_load_frames_device(self._h, C.c_void_p(dev_ptr), first, count))

    # -- stages
    def forward(self) -> None:
        L.check(self._lib.mc_plan_forward(self._h))

    def pairs(self) -> None:
        L.check(self._lib.mc_plan_pairs(self._h))

    def solve(self) -> None:
        L.check(self._lib.mc_plan_solve(self._h))

    def iterate(self) -> None:
        L.check(self._lib.mc_plan_iterate(self._h))

    def sum(self, want_image: bool = True) -> Optional[np.ndarray]:
        img = np.empty((self.nsam, self.nsam), dtype=np.float32) if want_image else None
        L.check(self._lib.mc_plan_sum(self._h, _ptr(img) if want_image else None))
        return img

    def run(self, want_image: bool = True, out: Optional[np.ndarray] = None) -> Optional[np.ndarray]:
        img = out if out is not None else (np.empty((self.nsam, self.nsam), dtype=np.float32) if want_image else None)
        L.check(self._lib.mc_plan_run(self._h, _ptr(img) if img is not None else None))
        return img

    def run_host(self, frames: np.ndarray, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Whole path from host frames (all positions) with the upload
        overlapped with the forward transforms (mc_plan_run_host)."""
        a = np.ascontiguousarray(frames)
        if a.dtype.itemsize != _WORD_LENGTH[self.info["mode"]] or a.shape[0] != self.nframe:
            raise ValueError("frames must hold every position in the plan's pixel type")
        img = out if out is not None else np.empty((self.nsam, self.nsam), dtype=np.float32)
        L.check(self._lib.mc_plan_run_host(self._h, _ptr(a), _ptr(img)))
        return img

    # -- extra sum-stage outputs (-srs, -2es, -ssc) and the exact count sum
    def raw_sum(self) -> np.ndarray:
        img = np.empty((self.nsam, self.nsam), dtype=np.float32)
        L.check(self._lib.mc_plan_raw_sum(self._h, _ptr(img)))
        return img

    def sum_to(self, last_frame: int) -> np.ndarray:
        img = np.empty((self.nsam, self.nsam), dtype=np.float32)
        L.check(self._lib.mc_plan_sum_to(self._h, last_frame, _ptr(img)))
        return img

    def corrected_frame(self, frame: int) -> np.ndarray:
        img = np.empty((self.nsam, self.nsam), dtype=np.float32)
        L.check(self._lib.mc_plan_corrected_frame(self._h, frame, _ptr(img)))
        return img

    QUICKLOOK = {"raw_fft": 0, "corr_sum": 1, "corr_fft": 2}

    def quicklook(self, which: str) -> np.ndarray:
        """-dsp 1 display (400 x 400 int16, 0..255): "raw_fft", "corr_sum" or "corr_fft"."""
        out = np.empty((400, 400), dtype=np.int16)
        L.check(self._lib.mc_plan_quicklook(self._h, self.QUICKLOOK[which], _ptr(out)))
        return out

    def fsc(self) -> np.ndarray:
        """-fsc table (nbox, 5): Nq%, D_Raw, U_Raw, D_Corr, U_Corr."""
        n = self.nsam
        nbox = (n // 2 + 1) // max(1, n // 400) + 1
        out = np.empty((nbox, 5), dtype=np.float64)
        nb = C.c_int()
        L.check(self._lib.mc_plan_fsc(self._h, _ptr(out), nbox, C.byref(nb)))
        return out[:nb.value]

    def count_sum(self) -> np.ndarray:
        nu = self.info["nsam_unbin"]
        out = np.empty((nu, nu), dtype=np.int32)
        L.check(self._lib.mc_plan_count_sum(self._h, _ptr(out)))
        return out

    # -- results
    def frame_shifts(self) -> np.ndarray:
        xy = np.empty((self.nframe, 2), dtype=np.float64)
        L.check(self._lib.mc_plan_get_frame_shifts(self._h, _ptr(xy)))
        return xy

    def pair_results(self) -> dict:
        P = self.npairs
        ij = np.empty((P, 2), dtype=np.int32)
        sh = np.empty((P, 2), dtype=np.float32)
        cc = np.empty(P, dtype=np.float32)
        pk = np.empty((P, 2), dtype=np.int32)
        L.check(self._lib.mc_plan_get_pairs(self._h, _ptr(ij), _ptr(sh), _ptr(cc), _ptr(pk)))
        return {"pairs": ij, "shift": sh, "cc": cc, "peak": pk}

    def ki(self) -> dict:
        P = self.npairs
        ki1 = np.empty(P, dtype=np.float64)
        kept = np.empty(P, dtype=np.int32)
        ki2 = np.empty(P, dtype=np.float64)
        nk = C.c_int()
        L.check(self._lib.mc_plan_get_ki(self._h, _ptr(ki1), C.byref(nk), _ptr(kept), _ptr(ki2)))
        return {"ki1": ki1, "kept": kept[: nk.value].copy(), "ki2": ki2[: nk.value].copy()}

    def frame_means(self) -> np.ndarray:
        m = np.empty(self.nframe, dtype=np.float32)
        L.check(self._lib.mc_plan_get_frame_means(self._h, _ptr(m)))
        return m

    def spectrum(self, pos: int, set_: int = 0) -> np.ndarray:
        """Half spectrum of position ``pos`` in the reference layout (ky rows, kx columns)."""
        n = self.nsam
        h = n // 2 + 1
        s = np.empty((h, n), dtype=np.complex64)
        L.check(self._lib.mc_plan_get_spectrum(self._h, set_, pos, _ptr(s)))
        return s.T.copy()

    def boxes(self) -> np.ndarray:
        b = self.params.CCPeakSearchDim
        out = np.empty((self.npairs, b, b), dtype=np.float32)
        L.check(self._lib.mc_plan_get_boxes(self._h, _ptr(out)))
        return out

    def sum_shifts(self) -> tuple[np.ndarray, int, int]:
        xy = np.empty((self.nframe, 2), dtype=np.float64)
        f, l = C.c_int(), C.c_int()
        L.check(self._lib.mc_plan_get_sum_shifts(self._h, _ptr(xy), C.byref(f), C.byref(l)))
        return xy, f.value, l.value

    def timings(self) -> dict:
        t = L.McTimings()
        L.check(self._lib.mc_plan_get_timings(self._h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in L.McTimings._fields_}

    def objective(self, shifts: np.ndarray) -> tuple[float, np.ndarray, np.ndarray]:
        """Frame-to-sum objective J at sum shifts (nframe, 2), its gradient
        (nframe, 2) from the adjoint kernel and the Hessian blocks (nframe, 3)."""
        s = np.ascontiguousarray(shifts, dtype=np.float64).reshape(self.nframe, 2)
        J = C.c_double()
        g = np.empty((self.nframe, 2))
        h = np.empty((self.nframe, 3))
        L.check(self._lib.mc_plan_objective(self._h, _ptr(s), C.byref(J), _ptr(g), _ptr(h)))
        return J.value, g, h

    def refine(self, iterations: int = 4) -> None:
        L.check(self._lib.mc_plan_refine(self._h, iterations))

    def set_profiling(self, on: bool) -> None:
        self._lib.mc_plan_set_profiling(self._h, int(on))

    def reset_stats(self) -> None:
        L.check(self._lib.mc_plan_reset_stats(self._h))

    def kernel_stats(self) -> dict:
        """{kernel name: {"ms", "launches", "bytes"}} accumulated since reset."""
        out = {}
        for k in range(KERNEL_KINDS):
            ms, n, b = C.c_double(), C.c_longlong(), C.c_double()
            L.check(self._lib.mc_plan_kernel_stats(self._h, k, C.byref(ms), C.byref(n), C.byref(b)))
            out[self._lib.mc_kernel_name(k).decode()] = {"ms": ms.value, "launches": n.value, "bytes": b.value}
        return out


def solve_pairs(nframe: int, pairs: np.ndarray, shifts: np.ndarray, kithresh: float = 1.0) -> dict:
    """Host FP64 drift solve (mc_solve_pairs): lsSolver + OD_Threshold + lsSolver."""
    ij = np.ascontiguousarray(pairs, dtype=np.int32)
    sh = np.ascontiguousarray(shifts, dtype=np.float32)
    P = ij.shape[0]
    step = np.empty((nframe - 1, 2))
    ki1 = np.empty(P)
    kept = np.empty(P, dtype=np.int32)
    ki2 = np.empty(P)
    nk = C.c_int()
    L.check(L.lib().mc_solve_pairs(nframe, P, _ptr(ij), _ptr(sh), kithresh, _ptr(step), _ptr(ki1),
                                   C.byref(nk), _ptr(kept), _ptr(ki2)))
    return {"step": step, "ki1": ki1, "kept": kept[: nk.value].copy(), "ki2": ki2[: nk.value].copy()}


def schedule_set(n: int, pair_q: int = 0, pairs_per_cta: int = 0, pair_variant: int = 0, fwd_streams: int = 0,
                 fwd_rows_pairing: int = 0, fwd_cols_pairing: int = 0) -> None:
    """Schedule for binned side n, used by plans created afterwards: the pair
    stage's split and pairs per CTA, the forward transforms' forked streams
    and radix-53 pairing of the row / column passes (0 = built-in)."""
    L.check(L.lib().mc_schedule_set(C.byref(L.McSchedule(n, pair_q, pairs_per_cta, pair_variant, fwd_streams,
                                                         fwd_rows_pairing, fwd_cols_pairing))))


def schedule_get(n: int) -> Optional[dict]:
    s = L.McSchedule()
    if L.lib().mc_schedule_get(n, C.byref(s)) != L.MC_OK:
        return None
    return {f: getattr(s, f) for f, _ in L.McSchedule._fields_}


def schedule_clear() -> None:
    L.lib().mc_schedule_clear()


def schedule_candidates(n: int) -> list[int]:
    """Codelet lengths Q the pair column stage takes for side n."""
    cnt = L.lib().mc_schedule_candidates(n, None, 0)
    q = (C.c_int * max(cnt, 1))()
    L.lib().mc_schedule_candidates(n, q, cnt)
    return list(q[:cnt])


class Batch:
    """Many movies on one GPU (mc_batch_*): `lanes` worker threads, each with
    its own stream and plans reused across movies of a geometry."""

    def __init__(self, device: int = 0, lanes: int = 2, graph: bool = False):
        """graph=True: each run is captured into one CUDA graph and launched
        once (mc_batch_set_graph; device frames, -itr 0, pinned or device
        images)."""
        self._lib = L.lib()
        _load_schedules()
        h = C.c_void_p()
        L.check(self._lib.mc_batch_create(device, lanes, C.byref(h)))
        self._h = h
        self.device = device
        self.lanes = lanes
        if graph:
            L.check(self._lib.mc_batch_set_graph(h, 1))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def device_bytes(self) -> int:
        return int(self._lib.mc_batch_device_bytes(self._h))

    def run(self, movies: list[dict], check: bool = True) -> list[dict]:
        """movies: dicts with `params` (verified Params), `nx`, `ny`, `nz`,
        `mode` and either `frames` (host array of the run's positions) or
        `device_ptr` (device address of them); optional `image` (float32
        nsam x nsam) and `frame_shifts` (float64 nframe x 2) outputs.
        Returns per movie: status, nsam, nframe, npairs, lane, start_ms,
        end_ms, gpu_ms, message."""
        n = len(movies)
        jobs = (L.McBatchJob * max(n, 1))()
        res = (L.McBatchResult * max(n, 1))()
        keep = []
        for i, m in enumerate(movies):
            j = jobs[i]
            if "device_ptr" in m:
                j.frames = C.c_void_p(int(m["device_ptr"]))
                j.on_device = 1
            else:
                a = np.ascontiguousarray(m["frames"])
                keep.append(a)
                j.frames = C.c_void_p(a.ctypes.data)
                j.on_device = 0
            j.nx, j.ny, j.nz, j.mode = m["nx"], m["ny"], m["nz"], m["mode"]
            j.params = m["params"].to_c()
            for key in ("image", "frame_shifts"):
                arr = m.get(key)
                if arr is not None:
                    want = np.float32 if key == "image" else np.float64
                    if arr.dtype != want or not arr.flags["C_CONTIGUOUS"]:
                        raise ValueError(f"{key} must be a C-contiguous {np.dtype(want).name} array")
                    setattr(j, key, C.c_void_p(arr.ctypes.data))
        rc = self._lib.mc_batch_run(self._h, jobs, n, res)
        out = []
        for i in range(n):
            r = res[i]
            out.append({"status": r.status, "nsam": r.nsam, "nframe": r.nframe, "npairs": r.npairs,
                        "lane": r.lane, "start_ms": r.start_ms, "end_ms": r.end_ms, "gpu_ms": r.gpu_ms,
                        "message": r.message.decode(errors="replace")})
        if check and rc != L.MC_OK:
            bad = next(o for o in out if o["status"] != L.MC_OK)
            raise L.McError(rc, bad["message"])
        return out


_PIXEL_DTYPE = {0: np.int8, 1: np.int16, 2: np.float32, 6: np.uint16, MODE_U8: np.uint8, MODE_F16: np.float16}
STACK_FORMATS = {0: "mrc", 1: "mrc-gz", 2: "tiff"}


class Stack:
    """A movie stack file (MRC, MRC-gz or strip TIFF) through mc_stack_*:
    the host-side readers MRC/MRCZ/MRCT and their detection order
    (DFAlign.cu:470-479).  Needs no GPU."""

    def __init__(self, path: str):
        self._lib = L.lib()
        h = C.c_void_p()
        L.check(self._lib.mc_stack_open(os.fsencode(path), C.byref(h)))
        self._h = h
        i = L.McStackInfo()
        L.check(self._lib.mc_stack_get_info(self._h, C.byref(i)))
        self.info = {k: getattr(i, k) for k, _ in L.McStackInfo._fields_}
        self.info["format_name"] = STACK_FORMATS[i.format]
        self.nx, self.ny, self.nz, self.mode = i.nx, i.ny, i.nz, i.mode

    def close(self) -> None:
        if self._h:
            self._lib.mc_stack_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def read_frames(self, first: int = 0, count: Optional[int] = None) -> np.ndarray:
        """Raw pixels (count, ny, nx) in the plan's pixel type for `mode`."""
        count = self.nz - first if count is None else count
        out = np.empty((count, self.ny, self.nx), dtype=_PIXEL_DTYPE[self.mode])
        got = C.c_int()
        L.check(self._lib.mc_stack_read_frames(self._h, _ptr(out), first, count, C.byref(got)))
        return out

    def read_frame_float(self, n: int) -> np.ndarray:
        out = np.empty((self.ny, self.nx), dtype=np.float32)
        L.check(self._lib.mc_stack_read_frame_float(self._h, _ptr(out), n))
        return out


def fft1d(d_in: int, d_out: int, n: int, batch: int, inverse: bool, stream: int = 0) -> None:
    """Engine transform on device pointers (tests)."""
    L.check(L.lib().mc_fft1d(n, batch, int(inverse), C.c_void_p(d_in), C.c_void_p(d_out),
                              C.c_void_p(stream) if stream else None))


def align(frames: np.ndarray, mode: int, params: Params, nz: Optional[int] = None,
          refs: Optional[dict] = None, log=None, stretch: Optional[tuple] = None,
          spectrum_slots: Optional[int] = None) -> dict:
    """Whole path on a stack already in host memory: frames (nz, ny, nx) in
    the file's pixel type.  Returns shifts, pair results and the sum."""
    nf, ny, nx = frames.shape
    nz = nz if nz is not None else nf
    with Plan(params, nx, ny, nz, mode, log=log, spectrum_slots=spectrum_slots) as pl:
        if stretch:
            pl.set_stretch(*stretch)
        if refs:
            pl.set_refs(**refs)
        pl.load_frames(frames[pl.info["nstart"]: pl.info["nend"] + 1])
        img = pl.run()
        return {"image": img, "frame_shifts": pl.frame_shifts(), **pl.pair_results(), **pl.ki(),
                "frame_mean": pl.frame_means(), "info": dict(pl.info), "timings": pl.timings()}
