"""Loaders for the reference's own code compiled by `make -C oracle ref`.

The shared objects live in oracle/_ref/ (not in git; they travel with the
repository snapshot).  Each loader returns None when its file is absent, so
callers skip rather than fail on a machine that never compiled them.

* run2_lib()   -- Optimizer::run2 (src/optimize.h:96-154) over DArray<double>
* ref_run2()   -- drive it with Python gradient / objective callbacks
* gpu_lib()    -- the reference's GPU build (exact-NUDFT stand-in for
                  cuFINUFFT) with the C entry points of
                  oracle/refgpu/ref_gpu_shim.cu
* ref_module() -- the reference's own Python module cTomocam
                  (src/pyTomocam.cpp) linked against that build
"""
from __future__ import annotations

import ctypes
import glob
import importlib.util
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

_GRAD = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                         ctypes.c_int64)
_ERR = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.c_int64)

_cache: dict = {}


def run2_lib():
    path = os.path.join(REF, "libref_run2.so")
    if not os.path.exists(path):
        return None
    if "run2" not in _cache:
        lib = ctypes.CDLL(path)
        lib.ref_run2.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_double, _GRAD, _ERR]
        lib.ref_run2.restype = ctypes.c_int
        _cache["run2"] = lib
    return _cache["run2"]


def ref_run2(x0, num_iters, step, grad_fn, err_fn):
    """Run the reference's run2 from x0 [S,R,C] (FP64).

    Returns (result, attempts, err_calls): attempts = gradient evaluations,
    err_calls = every objective value the reference asked for, in order.
    """
    lib = run2_lib()
    if lib is None:
        return None
    shape = x0.shape
    sol = np.ascontiguousarray(x0, dtype=np.float64).copy()
    counts = {"grad": 0}
    errs = []

    def g_cb(yp, gp, n):
        y = np.ctypeslib.as_array(yp, shape=(n,)).reshape(shape)
        g = np.ctypeslib.as_array(gp, shape=(n,))
        g[:] = np.asarray(grad_fn(y.copy()), dtype=np.float64).reshape(-1)
        counts["grad"] += 1

    def e_cb(xp, n):
        x = np.ctypeslib.as_array(xp, shape=(n,)).reshape(shape)
        e = float(err_fn(x.copy()))
        errs.append(e)
        return e

    gcb, ecb = _GRAD(g_cb), _ERR(e_cb)
    rc = lib.ref_run2(sol.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), shape[0], shape[1],
                      shape[2], int(num_iters), float(step), gcb, ecb)
    assert rc == 0
    return sol, counts["grad"], np.array(errs)


def gpu_lib():
    path = os.path.join(REF, "libref_gpu.so")
    if not os.path.exists(path):
        return None
    if "gpu" not in _cache:
        lib = ctypes.CDLL(path)
        fp = ctypes.POINTER(ctypes.c_float)
        vp = ctypes.c_void_p
        i, f, l = ctypes.c_int, ctypes.c_float, ctypes.c_long
        ip = ctypes.POINTER(ctypes.c_int)
        sig = {
            "ref_num_gpus": ([], i),
            "ref_preproc": ([fp, i, i, i, f, fp, l, ip], i),
            "ref_postproc": ([fp, i, i, i, fp, l, ip], i),
            "ref_pad2d": ([fp, i, i, i, i, fp, l, ip], i),
            "ref_roll": ([fp, fp, i, i, i, i], i),
            "ref_pad1d": ([fp, fp, i, i, i, i, i], i),
            "ref_qggmrf_dev": ([vp, vp, i, i, i, f, f], i),
            "ref_psf_create": ([fp, i, i, i, ctypes.POINTER(vp)], i),
            "ref_psf_destroy": ([vp], None),
            "ref_psf_grad_dev": ([vp, vp, vp, vp, i], i),
            "ref_gradient2_host": ([vp, fp, fp, fp, i], i),
            "ref_function_value2_host": ([vp, fp, fp, i, f], ctypes.c_double),
            "ref_add_total_var2_host": ([fp, fp, i, i, f, f], i),
            "ref_run2_host": ([vp, fp, fp, i, f, f, f, i, f], i),
            "ref_standin_stage": ([i, ctypes.c_int64, ctypes.c_int64, i, i, vp, ctypes.c_size_t],
                                  i),
            "ref_standin_clear": ([], None),
            "ref_standin_counts": ([ctypes.POINTER(l), ctypes.POINTER(l)], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _cache["gpu"] = lib
    return _cache["gpu"]


def fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def ref_module():
    """The reference's cTomocam module, imported as oracle._ref.cTomocam."""
    hits = glob.glob(os.path.join(REF, "cTomocam*.so"))
    if not hits or gpu_lib() is None:
        return None
    name = "oracle._ref.cTomocam"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, hits[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sys.modules[name] = mod
    return mod
