"""ctypes binding of libmc.so (include/mc.h).

The shared library is the product: this module only declares its C
signatures.  Importing fails loudly when libmc.so has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmc.so")

MC_OK = 0
ERRORS = {-1: "MC_E_ARG", -2: "MC_E_CUDA", -3: "MC_E_NOMEM", -4: "MC_E_SIZE", -5: "MC_E_STATE",
          -6: "MC_E_NUMERIC", -7: "MC_E_IO"}


class McParams(C.Structure):
    _fields_ = [
        ("crop_offsetx", C.c_int), ("crop_offsety", C.c_int), ("crop_nsam", C.c_int),
        ("bin", C.c_float),
        ("nStart", C.c_int), ("nEnd", C.c_int), ("nStartSum", C.c_int), ("nEndSum", C.c_int),
        ("GPUNum", C.c_int),
        ("bfactor", C.c_float), ("CCPeakSearchDim", C.c_int), ("FrameDistOffset", C.c_int),
        ("NoisePeakSize", C.c_int), ("kiThresh", C.c_float), ("bAlignToMid", C.c_int),
        ("iter", C.c_int), ("iterthres", C.c_float), ("refine", C.c_int),
    ]


class McInfo(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("mode", C.c_int),
        ("nsam_unbin", C.c_int), ("nsam", C.c_int),
        ("nstart", C.c_int), ("nend", C.c_int), ("nframe", C.c_int),
        ("npairs", C.c_int), ("two_sets", C.c_int), ("prune_p", C.c_int), ("prune_q", C.c_int),
        ("device_bytes", C.c_size_t), ("spectrum_slots", C.c_int), ("forward_recomputes", C.c_longlong),
    ]


class McTimings(C.Structure):
    _fields_ = [("forward_ms", C.c_float), ("pairs_ms", C.c_float), ("solve_ms", C.c_float),
                ("iterate_ms", C.c_float), ("sum_ms", C.c_float), ("total_ms", C.c_float),
                ("refine_ms", C.c_float)]


class McSchedule(C.Structure):
    _fields_ = [("n", C.c_int), ("pair_q", C.c_int), ("pairs_per_cta", C.c_int), ("pair_variant", C.c_int),
                ("fwd_streams", C.c_int), ("fwd_rows_pairing", C.c_int), ("fwd_cols_pairing", C.c_int)]


class McBatchJob(C.Structure):
    _fields_ = [("frames", C.c_void_p), ("on_device", C.c_int),
                ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("mode", C.c_int),
                ("params", McParams), ("image", C.c_void_p), ("frame_shifts", C.c_void_p)]


class McBatchResult(C.Structure):
    _fields_ = [("status", C.c_int), ("nsam", C.c_int), ("nframe", C.c_int), ("npairs", C.c_int),
                ("lane", C.c_int), ("start_ms", C.c_double), ("end_ms", C.c_double), ("gpu_ms", C.c_float),
                ("message", C.c_char * 160)]


class McStackInfo(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("mode", C.c_int), ("file_mode", C.c_int),
                ("format", C.c_int), ("bits", C.c_int), ("compression", C.c_int)]


LOG_FN = C.CFUNCTYPE(None, C.c_char_p, C.c_void_p)

# name -> (restype, argtypes)
SIGNATURES = {
    "mc_version": (C.c_int, []),
    "mc_strerror": (C.c_char_p, [C.c_int]),
    "mc_last_error": (C.c_char_p, []),
    "mc_debug_fail_alloc": (None, [C.c_int]),
    "mc_debug_device_budget": (None, [C.c_size_t]),
    "mc_default_params": (None, [C.POINTER(McParams)]),
    "mc_verify_params": (C.c_int, [C.POINTER(McParams), C.c_int]),
    "mc_plan_create": (C.c_int, [C.POINTER(McParams), C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mc_plan_destroy": (None, [C.c_void_p]),
    "mc_plan_info": (C.c_int, [C.c_void_p, C.POINTER(McInfo)]),
    "mc_plan_stream": (C.c_void_p, [C.c_void_p]),
    "mc_plan_set_log": (None, [C.c_void_p, LOG_FN, C.c_void_p]),
    "mc_plan_set_refs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mc_plan_load_frames": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "mc_plan_load_frames_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "mc_plan_forward": (C.c_int, [C.c_void_p]),
    "mc_plan_pairs": (C.c_int, [C.c_void_p]),
    "mc_plan_solve": (C.c_int, [C.c_void_p]),
    "mc_plan_iterate": (C.c_int, [C.c_void_p]),
    "mc_plan_sum": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc_plan_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc_plan_run_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mc_plan_get_frame_shifts": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc_plan_get_pairs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mc_plan_get_ki": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_void_p]),
    "mc_plan_get_frame_means": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc_plan_get_spectrum": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "mc_plan_get_boxes": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc_plan_get_sum_shifts": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mc_plan_get_timings": (C.c_int, [C.c_void_p, C.POINTER(McTimings)]),
    "mc_plan_set_profiling": (None, [C.c_void_p, C.c_int]),
    "mc_plan_reset_stats": (C.c_int, [C.c_void_p]),
    "mc_plan_kernel_stats": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_double)]),
    "mc_kernel_name": (C.c_char_p, [C.c_int]),
    "mc_plan_objective": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p, C.c_void_p]),
    "mc_plan_refine": (C.c_int, [C.c_void_p, C.c_int]),
    "mc_solve_pairs": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p,
                                 C.POINTER(C.c_int), C.c_void_p, C.c_void_p]),
    "mc_pair_window_static": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p,
                                        C.c_void_p]),
    "mc_fft1d": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mc_plan_raw_sum": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc_plan_sum_to": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "mc_plan_corrected_frame": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "mc_plan_count_sum": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc_plan_quicklook": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "mc_plan_fsc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "mc_plan_set_stretch": (C.c_int, [C.c_void_p, C.c_float, C.c_float]),
    "mc_plan_reframe": (C.c_int, [C.c_void_p, C.POINTER(McParams), C.c_int]),
    "mc_plan_create_capacity": (C.c_int, [C.POINTER(McParams), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.POINTER(C.c_void_p)]),
    "mc_plan_create_slots": (C.c_int, [C.POINTER(McParams), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mc_plan_bind_frames_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc_schedule_set": (C.c_int, [C.POINTER(McSchedule)]),
    "mc_schedule_get": (C.c_int, [C.c_int, C.POINTER(McSchedule)]),
    "mc_schedule_clear": (None, []),
    "mc_schedule_candidates": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.c_int]),
    "mc_batch_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mc_batch_destroy": (None, [C.c_void_p]),
    "mc_batch_run": (C.c_int, [C.c_void_p, C.POINTER(McBatchJob), C.c_int, C.POINTER(McBatchResult)]),
    "mc_batch_device_bytes": (C.c_size_t, [C.c_void_p]),
    "mc_batch_set_graph": (C.c_int, [C.c_void_p, C.c_int]),
    "mc_stack_open": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mc_stack_get_info": (C.c_int, [C.c_void_p, C.POINTER(McStackInfo)]),
    "mc_stack_read_frames": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "mc_stack_read_frame_float": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "mc_stack_close": (None, [C.c_void_p]),
}


class McError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libmc.so not built ({LIB_PATH}); run python -m motioncorr1exp_b200.build")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != MC_OK:
        raise McError(code, lib().mc_last_error().decode(errors="replace"))
