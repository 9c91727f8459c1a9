"""ctypes binding of the C ABI in ``include/tomocam_b200.h``.

This is the thin layer the torch paths and the tests use to reach the CUDA
library with device pointers.  Every call is checked; a non-zero status
raises ``TomocamError`` carrying ``tc_last_error_string()``.  Loading fails
loudly when the shared library has not been built: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtomocam_b200.so")

TC_OK = 0
TC_ERR_ARG = -1
TC_ERR_SHAPE = -2
TC_ERR_ALLOC = -3
TC_ERR_CUDA = -4
TC_ERR_TIMEOUT = -5
TC_ERR_NAN = -6
TC_ERR_STATE = -7
TC_PLAN_NO_PSF = 1
TC_PLAN_AUTOTUNE = 2
TC_PLAN_POW2_TOEPLITZ = 4
TC_PLAN_UNPAIRED = 8

_ERR_NAMES = {
    TC_ERR_ARG: "TC_ERR_ARG", TC_ERR_SHAPE: "TC_ERR_SHAPE", TC_ERR_ALLOC: "TC_ERR_ALLOC",
    TC_ERR_CUDA: "TC_ERR_CUDA", TC_ERR_TIMEOUT: "TC_ERR_TIMEOUT", TC_ERR_NAN: "TC_ERR_NAN",
    TC_ERR_STATE: "TC_ERR_STATE",
}


class TomocamError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Geom(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("nproj", ctypes.c_int32),
                ("angles", ctypes.POINTER(ctypes.c_float)), ("nufft_tol", ctypes.c_double),
                ("max_batch", ctypes.c_int32), ("flags", ctypes.c_int32)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("nproj", ctypes.c_int32), ("nf", ctypes.c_int32),
                ("kernel_width", ctypes.c_int32), ("toeplitz_m", ctypes.c_int32),
                ("max_batch", ctypes.c_int32), ("workspace_bytes", ctypes.c_int64),
                ("table_bytes", ctypes.c_int64), ("lipschitz", ctypes.c_double),
                ("toeplitz_pairs", ctypes.c_int32), ("toeplitz_fast", ctypes.c_int32),
                ("spread_tile", ctypes.c_int32), ("spread_max_points", ctypes.c_int32),
                ("band_chunk", ctypes.c_int32), ("interp_tile", ctypes.c_int32),
                ("interp_max_points", ctypes.c_int32), ("paired_nufft", ctypes.c_int32)]


class MbirOpts(ctypes.Structure):
    _fields_ = [("num_iters", ctypes.c_int32), ("sigma", ctypes.c_float), ("p", ctypes.c_float),
                ("prior_weight", ctypes.c_float), ("step", ctypes.c_float),
                ("use_graph", ctypes.c_int32), ("max_attempts", ctypes.c_int32),
                ("verbose", ctypes.c_int32), ("phase_ms", ctypes.c_void_p)]


class Scan(ctypes.Structure):
    _fields_ = [("plan", ctypes.c_void_p), ("aty", ctypes.c_void_p), ("sino_sq", ctypes.c_double),
                ("x", ctypes.c_void_p), ("nslices", ctypes.c_int32), ("sigma", ctypes.c_float),
                ("p", ctypes.c_float), ("prior_weight", ctypes.c_float), ("step", ctypes.c_float)]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); the tests check this table against the header
PROTOTYPES = {
    "tc_plan_create": (_i, [ctypes.POINTER(Geom), ctypes.POINTER(_vp)]),
    "tc_plan_destroy": (_i, [_vp]),
    "tc_plan_get_info": (_i, [_vp, ctypes.POINTER(PlanInfo)]),
    "tc_radon": (_i, [_vp, _vp, _vp, _i, _vp]),
    "tc_iradon": (_i, [_vp, _vp, _vp, _i, _i, _vp]),
    "tc_toeplitz_grad": (_i, [_vp, _vp, _vp, _vp, _i, _dp, _dp, _vp]),
    "tc_toeplitz_grad_noalloc": (_i, [_vp, _vp, _vp, _vp, _i, _dp, _dp, _vp]),
    "tc_nufft_grad": (_i, [_vp, _vp, _vp, _vp, _i, _vp]),
    "tc_qggmrf_grad": (_i, [_vp, _vp, _i, _i, _i, _f, _f, _f, _vp]),
    "tc_qggmrf_value": (_i, [_vp, _i, _i, _i, _f, _f, _dp, _dp, _vp]),
    "tc_qggmrf_hvp": (_i, [_vp, _vp, _vp, _i, _i, _i, _f, _f, _f, _dp, _dp, _vp]),
    "tc_plan_get_psf": (_i, [_vp, _dp]),
    "tc_plan_set_psf": (_i, [_vp, _dp]),
    "tc_fft_c2c": (_i, [_vp, _vp, _i, _i, _i, _vp]),
    "tc_axpby": (_i, [_f, _vp, _f, _vp, ctypes.c_size_t, _vp]),
    "tc_mbir_opts_default": (None, [ctypes.POINTER(MbirOpts)]),
    "tc_mbir_solve": (_i, [_vp, _vp, _d, _vp, _i, ctypes.POINTER(MbirOpts), _dp, _vp]),
    "tc_mbir_batched": (_i, [ctypes.POINTER(Scan), _i, _i, _i, _i, _dp, _vp]),
    "tc_slab_create": (_i, [_vp, _vp, _d, _vp, _i, ctypes.POINTER(MbirOpts), ctypes.POINTER(_vp), _vp]),
    "tc_slab_halo": (_i, [_vp, _i, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                          ctypes.POINTER(_vp), ctypes.POINTER(_i)]),
    "tc_slab_attempt": (_i, [_vp, ctypes.POINTER(_vp), _vp]),
    "tc_slab_decide": (_i, [_vp, ctypes.POINTER(_i), _vp]),
    "tc_slab_result": (_i, [_vp, _vp, _dp, ctypes.POINTER(_i), _vp]),
    "tc_slab_destroy": (_i, [_vp]),
    "tc_radon_host": (_i, [_fp, _i, _i, _fp, _i, _fp]),
    "tc_backproject_host": (_i, [_fp, _i, _i, _i, _fp, _f, _fp]),
    "tc_mbir_host": (_i, [_fp, _i, _i, _i, _fp, _f, _i, _f, _f, _f, _fp,
                          ctypes.POINTER(MbirOpts)]),
    "tc_sino_ingest_psd": (_i, [_fp, _i, _i, _i, _i, _i, _vp]),
    "tc_set_num_of_gpus": (_i, [_i]),
    "tc_last_error_string": (ctypes.c_char_p, []),
    "tc_version": (ctypes.c_char_p, []),
    "tc_release_cached_memory": (_i, []),
}

_LIB = None


def lib():
    """Load libtomocam_b200.so (once) and attach the prototypes."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m tomocam_b200.build` "
                "(the CUDA library is required; there is no CPU implementation)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc: int):
    if rc != TC_OK:
        msg = lib().tc_last_error_string()
        raise TomocamError(rc, msg.decode() if msg else "")
    return rc


def call(name: str, *args):
    return check(getattr(lib(), name)(*args))
