"""B200-native drift correction of dose-fractionated movies (MotionCorr 1 path).

The product is libmc.so (include/mc.h), hand-written sm_100a CUDA behind a C
ABI, and the dosefgpu_driftcorr CLI built on it.  This package holds the
sources, the in-tree build, a ctypes binding, MRC I/O and the synthetic
movie generator.
"""
from .api import Params, Plan, align, default_params, verify_params  # noqa: F401

__all__ = ["Params", "Plan", "align", "default_params", "verify_params"]
