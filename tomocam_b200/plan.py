"""Device-level API on torch CUDA tensors, over the C ABI.

``Plan`` owns a ``tc_plan`` (geometry, FP64 point-spread function, FFT
tables, workspace) and exposes the operators of the MBIR path on float32
CUDA tensors laid out like the reference's arrays: images ``[S, N, N]``,
sinograms ``[S, P, N]``.  All work is enqueued on torch's current stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the runtime image
    torch = None


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _check_tensor(t, shape, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.float32:
        raise TypeError(f"{name} must be float32")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")


class Plan:
    """Geometry of one scan: N x N images, ``len(angles)`` projections of N pixels."""

    def __init__(self, n: int, angles, nufft_tol: float = 0.0, max_batch: int = 0,
                 psf: bool = True, autotune: bool = False, pow2_toeplitz: bool = False,
                 paired: bool = True):
        """max_batch: slices per internal chunk (0: chosen by the plan; NUFFT
        chunks hold at most 16 slices when paired, 8 otherwise; Toeplitz
        chunks max(1, max_batch // 2) slice pairs).  pow2_toeplitz: a
        power-of-two Toeplitz FFT size, which mbir_batched
        needs for images of 513 .. 768 and 1025 .. 1536 pixels.  paired=False
        keeps one slice per complex line in the NUFFT operators (by default
        the register-FFT path carries two slices per line)."""
        self._h = ctypes.c_void_p()
        ang = np.ascontiguousarray(np.asarray(angles, dtype=np.float32).reshape(-1))
        self.angles = ang
        g = _lib.Geom(int(n), int(ang.size),
                      ang.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(nufft_tol),
                      int(max_batch), (0 if psf else _lib.TC_PLAN_NO_PSF) |
                      (_lib.TC_PLAN_AUTOTUNE if autotune else 0) |
                      (_lib.TC_PLAN_POW2_TOEPLITZ if pow2_toeplitz else 0) |
                      (0 if paired else _lib.TC_PLAN_UNPAIRED))
        _lib.call("tc_plan_create", ctypes.byref(g), ctypes.byref(self._h))
        self.n = int(n)
        self.nproj = int(ang.size)

    def close(self):
        if self._h:
            _lib.lib().tc_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

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
    def info(self) -> dict:
        inf = _lib.PlanInfo()
        _lib.call("tc_plan_get_info", self._h, ctypes.byref(inf))
        return {k: getattr(inf, k) for k, _ in inf._fields_}

    # ---- operators --------------------------------------------------------
    def radon(self, x, out=None):
        S = x.shape[0]
        _check_tensor(x, (S, self.n, self.n), "x")
        out = torch.empty((S, self.nproj, self.n), device=x.device, dtype=torch.float32) if out is None else out
        _check_tensor(out, (S, self.nproj, self.n), "out")
        _lib.call("tc_radon", self._h, _ptr(x), _ptr(out), S, _stream())
        return out

    def iradon(self, sino, ramp: bool = False, out=None):
        S = sino.shape[0]
        _check_tensor(sino, (S, self.nproj, self.n), "sino")
        out = torch.empty((S, self.n, self.n), device=sino.device, dtype=torch.float32) if out is None else out
        _check_tensor(out, (S, self.n, self.n), "out")
        _lib.call("tc_iradon", self._h, _ptr(sino), _ptr(out), S, int(bool(ramp)), _stream())
        return out

    def toeplitz_grad(self, x, aty=None, out=None, dots: bool = False):
        """g = H x - aty; with dots=True also returns (x.Hx, x.aty) in FP64."""
        S = x.shape[0]
        _check_tensor(x, (S, self.n, self.n), "x")
        if aty is not None:
            _check_tensor(aty, (S, self.n, self.n), "aty")
        out = torch.empty_like(x) if out is None else out
        _check_tensor(out, (S, self.n, self.n), "out")
        a = ctypes.c_double(0.0)
        b = ctypes.c_double(0.0)
        _lib.call("tc_toeplitz_grad", self._h, _ptr(x), _ptr(aty), _ptr(out), S,
                  ctypes.byref(a) if dots else None, ctypes.byref(b) if dots else None, _stream())
        return (out, a.value, b.value) if dots else out

    def nufft_grad(self, x, aty=None, out=None):
        S = x.shape[0]
        _check_tensor(x, (S, self.n, self.n), "x")
        if aty is not None:
            _check_tensor(aty, (S, self.n, self.n), "aty")
        out = torch.empty_like(x) if out is None else out
        _lib.call("tc_nufft_grad", self._h, _ptr(x), _ptr(aty), _ptr(out), S, _stream())
        return out

    def psf(self) -> np.ndarray:
        m = 2 * self.n - 1
        out = np.empty((m, m), dtype=np.float64)
        _lib.call("tc_plan_get_psf", self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def set_psf(self, psf):
        m = 2 * self.n - 1
        a = np.ascontiguousarray(np.asarray(psf, dtype=np.float64))
        if a.shape != (m, m):
            raise ValueError(f"psf must have shape ({m}, {m})")
        _lib.call("tc_plan_set_psf", self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def mbir_solve(self, aty, sino_sq: float, x0, num_iters: int, sigma: float, p: float = 1.2,
                   prior_weight: float = 1.0, step: float = 0.0, use_graph: bool = True,
                   max_attempts: int = 0, verbose: bool = False, inplace: bool = False,
                   phase_ms=None):
        """Run Optimizer::run2 on the device.

        Returns (x, history[num_iters, 3]): per iteration the objective, the
        step norm |x_k+1 - x_k| and the number of backtracking attempts.
        phase_ms (host float64 array of 4, host loop only) receives the summed
        device milliseconds of the update kernel, the Toeplitz passes and the
        step test, and the number of attempts.
        """
        S = x0.shape[0]
        _check_tensor(aty, (S, self.n, self.n), "aty")
        _check_tensor(x0, (S, self.n, self.n), "x0")
        x = x0 if inplace else x0.clone()
        o = _lib.MbirOpts()
        _lib.lib().tc_mbir_opts_default(ctypes.byref(o))
        o.num_iters, o.sigma, o.p, o.prior_weight = int(num_iters), float(sigma), float(p), float(prior_weight)
        o.step, o.use_graph, o.max_attempts, o.verbose = float(step), int(bool(use_graph)), int(max_attempts), int(bool(verbose))
        if phase_ms is not None:
            if not (isinstance(phase_ms, np.ndarray) and phase_ms.dtype == np.float64 and
                    phase_ms.size >= 4 and phase_ms.flags.c_contiguous):
                raise ValueError("phase_ms must be a contiguous float64 array of 4")
            o.phase_ms = phase_ms.ctypes.data
        hist = np.zeros((max(int(num_iters), 1), 3), dtype=np.float64)
        _lib.call("tc_mbir_solve", self._h, _ptr(aty), float(sino_sq), _ptr(x), S, ctypes.byref(o),
                  hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _stream())
        return x, hist[:int(num_iters)]


class BatchScan:
    """One scan of mbir_batched: its plan, A^T y, ||y||^2, image (in: initial
    guess; replaced by the result) and prior (sigma, p, prior weight beta)."""

    def __init__(self, plan: Plan, aty, sino_sq: float, x, sigma: float, p: float = 1.2,
                 prior_weight: float = 1.0, step: float = 0.0):
        S = x.shape[0]
        _check_tensor(aty, (S, plan.n, plan.n), "aty")
        _check_tensor(x, (S, plan.n, plan.n), "x")
        self.plan, self.aty, self.sino_sq, self.x = plan, aty, float(sino_sq), x
        self.sigma, self.p, self.prior_weight, self.step = float(sigma), float(p), float(prior_weight), float(step)


def mbir_batched(scans, num_iters: int, use_graph: bool = True, max_attempts: int = 0):
    """Solve independent scans of uneven sizes together (tc_mbir_batched):
    every scan runs Optimizer::run2 as mbir_solve would, and each attempt of
    all running scans is one launch per kernel.  The scans' x tensors are
    overwritten with the results; returns history[nscans, num_iters, 3]."""
    scans = list(scans)
    arr = (_lib.Scan * max(len(scans), 1))()
    for i, s in enumerate(scans):
        arr[i] = _lib.Scan(s.plan._h.value, s.aty.data_ptr(), s.sino_sq, s.x.data_ptr(),
                           int(s.x.shape[0]), s.sigma, s.p, s.prior_weight, s.step)
    K = int(num_iters)
    hist = np.zeros((max(len(scans), 1), max(K, 1), 3), dtype=np.float64)
    _lib.call("tc_mbir_batched", arr, len(scans), K, int(bool(use_graph)), int(max_attempts),
              hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _stream())
    return hist[:len(scans), :K]


def qggmrf_grad(x, g, sigma: float, p: float = 1.2, scale: float = 1.0):
    """In place: g += scale * qGGMRF'(x) on [S, R, C] CUDA tensors."""
    _check_tensor(x, None, "x")
    _check_tensor(g, tuple(x.shape), "g")
    if x.dim() != 3:
        raise ValueError("x must be [S, R, C]")
    S, R, C = x.shape
    _lib.call("tc_qggmrf_grad", _ptr(x), _ptr(g), S, R, C, float(sigma), float(p), float(scale),
              _stream())
    return g


def qggmrf_value(x, sigma: float, p: float = 1.2):
    """(U(x), dU/dsigma) in FP64 for the prior potential
    U = 1/2 sum_v sum_26 w rho(x_v - x_n) whose gradient qggmrf_grad adds."""
    _check_tensor(x, None, "x")
    if x.dim() != 3:
        raise ValueError("x must be [S, R, C]")
    S, R, C = x.shape
    u = ctypes.c_double(0.0)
    du = ctypes.c_double(0.0)
    _lib.call("tc_qggmrf_value", _ptr(x), S, R, C, float(sigma), float(p), ctypes.byref(u),
              ctypes.byref(du), _stream())
    return u.value, du.value


def qggmrf_hvp(x, v, sigma: float, p: float = 1.2, scale: float = 1.0, out=None,
               dots: bool = True):
    """Prior second-order terms at x along v: returns (hv, v.grad U, v.dgrad U/dsigma)
    with hv = scale * Hess U(x) v (dots None when dots=False)."""
    _check_tensor(x, None, "x")
    _check_tensor(v, tuple(x.shape), "v")
    if x.dim() != 3:
        raise ValueError("x must be [S, R, C]")
    S, R, C = x.shape
    out = torch.empty_like(x) if out is None else out
    _check_tensor(out, tuple(x.shape), "out")
    a = ctypes.c_double(0.0)
    b = ctypes.c_double(0.0)
    _lib.call("tc_qggmrf_hvp", _ptr(x), _ptr(v), _ptr(out), S, R, C, float(sigma), float(p),
              float(scale), ctypes.byref(a) if dots else None, ctypes.byref(b) if dots else None,
              _stream())
    return (out, a.value, b.value) if dots else (out, None, None)


def fft_c2c(x, direction: int = -1, out=None):
    """Unnormalised FFT along the last axis of a complex64 CUDA tensor."""
    if not (x.is_cuda and x.dtype == torch.complex64 and x.is_contiguous()):
        raise TypeError("x must be a contiguous complex64 CUDA tensor")
    n = x.shape[-1]
    nb = x.numel() // n if n else 0
    out = torch.empty_like(x) if out is None else out
    _lib.call("tc_fft_c2c", _ptr(x), _ptr(out), nb, n, int(direction), _stream())
    return out


def release_cached_memory():
    """Free the device memory the library keeps for reuse on the current
    device (tc_release_cached_memory): blocks of destroyed plans and of the
    host entry points' temporaries, kept up to half the device's memory."""
    _lib.call("tc_release_cached_memory")


def axpby(a: float, x, b: float, y):
    """In place: y = a x + b y."""
    _check_tensor(x, None, "x")
    _check_tensor(y, tuple(x.shape), "y")
    _lib.call("tc_axpby", ctypes.c_float(a), _ptr(x), ctypes.c_float(b), _ptr(y), x.numel(), _stream())
    return y
