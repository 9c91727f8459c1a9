"""FP64 CPU oracle for tomoCAM's MBIR path -- TEST INFRASTRUCTURE ONLY.

This module restates, in double precision, the algorithm that the reference
(lbl-camera/tomocam 3.0) runs for its MBIR path.  It is the checker for the
CUDA implementation in ``tomocam_b200``: only ``tests/``, the smoke check and
``bench.py``'s CPU-baseline / reference arm may import it.  The product never
routes through it.

Every function cites the reference file:line it follows (paths are relative
to the reference project root).

NUFFT boundary.  The reference computes its non-uniform FFTs with cuFINUFFT
(``src/nufft.h:196-384``), a third-party library that the reference does not
vendor or pin (``cmake/Findfinufft.cmake`` accepts any installed version).
Here the transforms are evaluated two ways:

* ``exact``: the direct non-uniform DFT -- the definition cuFINUFFT
  approximates (type 1, iflag +1 and type 2, iflag -1, x paired with the fast
  image axis, modes ``k = idx - n//2``).  Used at small sizes; exact to
  rounding.
* ``es``: the exponential-of-semicircle NUFFT of Barnett, Magland & af
  Klinteberg (SIAM J. Sci. Comput. 2019), upsampling 2, width
  ``ceil(log10(1/tol)) + 1``, ``beta = 2.30 * width``, deconvolution by the
  kernel's Fourier transform computed with Gauss-Legendre quadrature.  Used
  for large sizes; checked against ``exact`` in the tests.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field

import numpy as np

try:  # multithreaded FP64 FFTs when scipy is present
    import scipy.fft as _sfft

    def _fftn(a, axes, inverse=False):
        f = _sfft.ifftn if inverse else _sfft.fftn
        return f(a, axes=axes, workers=-1)

    def _fft(a, axis, inverse=False):
        f = _sfft.ifft if inverse else _sfft.fft
        return f(a, axis=axis, workers=-1)

    def _rfft2(a):
        return _sfft.rfft2(a, workers=-1)

    def _irfft2(a, s):
        return _sfft.irfft2(a, s=s, workers=-1)
except ImportError:  # pragma: no cover
    def _rfft2(a):
        return np.fft.rfft2(a)

    def _irfft2(a, s):
        return np.fft.irfft2(a, s=s)

    def _fftn(a, axes, inverse=False):
        return (np.fft.ifftn if inverse else np.fft.fftn)(a, axes=axes)

    def _fft(a, axis, inverse=False):
        return (np.fft.ifft if inverse else np.fft.fft)(a, axis=axis)


# --------------------------------------------------------------------------
# constants of the prior, src/gpu/potential_function.cuh:31-51.  The
# reference stores them as float; the float32-rounded values are used so the
# oracle evaluates the same function.
# --------------------------------------------------------------------------
MRF_Q = 2.0
MRF_C = float(np.float32(0.001))
_W = np.array([[[0.0302, 0.0370, 0.0302],
                [0.0370, 0.0523, 0.0370],
                [0.0302, 0.0370, 0.0302]],
               [[0.0370, 0.0523, 0.0370],
                [0.0523, 0.0000, 0.0523],
                [0.0370, 0.0523, 0.0370]],
               [[0.0302, 0.0370, 0.0302],
                [0.0370, 0.0523, 0.0370],
                [0.0302, 0.0370, 0.0302]]], dtype=np.float32)
QGGMRF_WEIGHTS = _W.astype(np.float64)

# --------------------------------------------------------------------------
# optional C accelerator (oracle/oracle_core.c)
# --------------------------------------------------------------------------
_HERE = os.path.dirname(os.path.abspath(__file__))
_CORE = None


def _core():
    global _CORE
    if _CORE is None:
        path = os.path.join(_HERE, "liboracle_core.so")
        if not os.path.exists(path):
            build_core()
        lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.orc_es_spread.argtypes = [ctypes.c_int64, dp, dp, dp, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_double, dp]
        lib.orc_es_interp.argtypes = [ctypes.c_int64, dp, dp, dp, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_double, dp]
        lib.orc_qggmrf.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   dp, ctypes.c_double]
        _CORE = lib
    return _CORE


def build_core(force: bool = False) -> str:
    """Compile oracle_core.c into oracle/liboracle_core.so (gcc, OpenMP)."""
    import subprocess
    src = os.path.join(_HERE, "oracle_core.c")
    out = os.path.join(_HERE, "liboracle_core.so")
    if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared",
                               "-o", out, src, "-lm"])
    return out


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# --------------------------------------------------------------------------
# geometry
# --------------------------------------------------------------------------
def polar_grid(nproj: int, ncols: int, angles):
    """Polar k-space points, src/gpu/nufft_utils.cu:32-44.

    r_j = 2*pi/(ncols-1) * (j - ncols//2);  x = r cos(theta), y = r sin(theta).
    Returns two [nproj, ncols] float64 arrays.
    """
    ang = np.asarray(angles, dtype=np.float64).reshape(-1)
    assert ang.size == nproj
    s = 2.0 * np.pi / (ncols - 1)
    r = s * (np.arange(ncols, dtype=np.float64) - (ncols // 2))
    return r[None, :] * np.cos(ang)[:, None], r[None, :] * np.sin(ang)[:, None]


def _modes(n):
    return np.arange(n, dtype=np.float64) - (n // 2)


# --------------------------------------------------------------------------
# non-uniform DFTs (the definition cuFINUFFT approximates)
# --------------------------------------------------------------------------
def nudft_type2(f, x, y):
    """c[s, j] = sum_{m2, m1} f[s, m2, m1] exp(-i (m1 x_j + m2 y_j)).

    Type 2, iflag -1 (src/nufft.h:311-346).  f: [S, n, n] complex; x, y:
    point arrays of any shape; returns [S, npts].
    """
    f = np.asarray(f, dtype=np.complex128)
    S, n2, n1 = f.shape
    xs = np.asarray(x, dtype=np.float64).reshape(-1)
    ys = np.asarray(y, dtype=np.float64).reshape(-1)
    ex = np.exp(-1j * np.outer(xs, _modes(n1)))      # [npts, n1]
    ey = np.exp(-1j * np.outer(ys, _modes(n2)))      # [npts, n2]
    out = np.empty((S, xs.size), dtype=np.complex128)
    for s in range(S):
        t = ey @ f[s]                                 # [npts, n1]
        out[s] = np.einsum("pm,pm->p", t, ex)
    return out


def nudft_type1(c, x, y, n1, n2=None):
    """f[s, m2, m1] = sum_j c[s, j] exp(+i (m1 x_j + m2 y_j)).

    Type 1, iflag +1 (src/nufft.h:230-267).  c: [S, npts] complex.
    Returns [S, n2, n1].
    """
    n2 = n1 if n2 is None else n2
    c = np.asarray(c, dtype=np.complex128)
    S = c.shape[0]
    xs = np.asarray(x, dtype=np.float64).reshape(-1)
    ys = np.asarray(y, dtype=np.float64).reshape(-1)
    ex = np.exp(1j * np.outer(xs, _modes(n1)))       # [npts, n1]
    ey = np.exp(1j * np.outer(ys, _modes(n2)))       # [npts, n2]
    out = np.empty((S, n2, n1), dtype=np.complex128)
    for s in range(S):
        out[s] = (ey * c[s][:, None]).T @ ex
    return out


# --------------------------------------------------------------------------
# ES-kernel NUFFT (published method; see module docstring)
# --------------------------------------------------------------------------
@dataclass
class ESParams:
    tol: float
    w: int = field(init=False)
    beta: float = field(init=False)

    def __post_init__(self):
        self.w = int(math.ceil(math.log10(1.0 / self.tol))) + 1
        self.beta = 2.30 * self.w


def _next_smooth(n):
    """smallest 2^a 3^b 5^c >= n"""
    best = None
    p2 = 1
    while p2 < 2 * n:
        p3 = p2
        while p3 < 2 * n:
            p5 = p3
            while p5 < 2 * n:
                if p5 >= n and (best is None or p5 < best):
                    best = p5
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return best


def es_fine_size(nmodes):
    nf = _next_smooth(2 * nmodes)
    return nf + (nf & 1)


def es_kernel_ft(k, nf, prm: ESParams):
    """psi_hat(k) = int psi(t) cos(k t) dt for psi(t) = phi(2t/(w h)), h = 2 pi/nf."""
    nodes, wts = np.polynomial.legendre.leggauss(4 * prm.w + 40)
    half = 0.5 * prm.w * (2.0 * np.pi / nf)
    phi = np.exp(prm.beta * (np.sqrt(1.0 - nodes ** 2) - 1.0))
    k = np.asarray(k, dtype=np.float64)
    return half * (np.cos(np.outer(k, nodes) * half) @ (wts * phi))


def es_type2(f, x, y, tol=1e-12):
    """ES-kernel approximation of nudft_type2."""
    prm = ESParams(tol)
    f = np.asarray(f, dtype=np.complex128)
    S, n2, n1 = f.shape
    assert n1 == n2
    n = n1
    nf = es_fine_size(n)
    m = _modes(n)
    corr = (2.0 * np.pi / nf) / es_kernel_ft(m, nf, prm)
    grid = np.zeros((S, nf, nf), dtype=np.complex128)
    idx = np.mod(m.astype(np.int64), nf)
    grid[:, idx[:, None], idx[None, :]] = f * corr[None, :, None] * corr[None, None, :]
    b = _fftn(grid, axes=(1, 2))
    xs = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    ys = np.ascontiguousarray(np.asarray(y, dtype=np.float64).reshape(-1))
    out = np.empty((S, xs.size), dtype=np.complex128)
    bb = np.ascontiguousarray(b)
    _core().orc_es_interp(xs.size, _dptr(xs), _dptr(ys), _dptr(bb.view(np.float64)),
                          S, nf, prm.w, prm.beta, _dptr(out.view(np.float64)))
    return out


def es_type1(c, x, y, n1, tol=1e-12):
    """ES-kernel approximation of nudft_type1 (square mode grid n1 x n1)."""
    prm = ESParams(tol)
    c = np.ascontiguousarray(np.asarray(c, dtype=np.complex128))
    S = c.shape[0]
    nf = es_fine_size(n1)
    xs = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    ys = np.ascontiguousarray(np.asarray(y, dtype=np.float64).reshape(-1))
    grid = np.empty((S, nf, nf), dtype=np.complex128)
    _core().orc_es_spread(xs.size, _dptr(xs), _dptr(ys), _dptr(c.view(np.float64)),
                          S, nf, prm.w, prm.beta, _dptr(grid.view(np.float64)))
    a = _fftn(grid, axes=(1, 2), inverse=True) * (nf * nf)
    m = _modes(n1)
    idx = np.mod(m.astype(np.int64), nf)
    corr = (2.0 * np.pi / nf) / es_kernel_ft(m, nf, prm)
    return a[:, idx[:, None], idx[None, :]] * corr[None, :, None] * corr[None, None, :]


def nufft_type2(f, x, y, method="exact", tol=1e-12):
    return nudft_type2(f, x, y) if method == "exact" else es_type2(f, x, y, tol)


def nufft_type1(c, x, y, n1, method="exact", tol=1e-12):
    return nudft_type1(c, x, y, n1) if method == "exact" else es_type1(c, x, y, n1, tol)


# --------------------------------------------------------------------------
# radon / back-projection on one device
# --------------------------------------------------------------------------
def project(img, angles, method="exact", tol=1e-12):
    """Forward projection A x, src/forward.cpp:34-52.

    radon = Re(fftshift(IFFT(ifftshift(NUFFT2(x)))))/N^2 along the detector
    axis, with the unnormalised inverse FFT (cuFFT INVERSE, src/fft.h:131-151)
    and numpy shift semantics (src/gpu/fftshift.cuh:60-83, fftshift.cu:30-40).
    img: [S, N, N] -> [S, P, N].
    """
    img = np.asarray(img, dtype=np.float64)
    S, N, N2 = img.shape
    assert N == N2
    P = len(angles)
    x, y = polar_grid(P, N, angles)
    c = nufft_type2(img.astype(np.complex128), x, y, method, tol).reshape(S, P, N)
    c = np.fft.ifftshift(c, axes=-1)
    c = _fft(c, axis=-1, inverse=True) * N
    c = np.fft.fftshift(c, axes=-1)
    return c.real / float(N * N)


def ramp_filter(ncols):
    """Ram-Lak weights |k - n//2| / n on the centred spectrum, src/gpu/ramlak.cu:15-31."""
    freq = np.abs(np.arange(ncols, dtype=np.float64) - float(ncols // 2)) / float(ncols)
    return np.where(freq < 1.0, freq, 0.0)


def backproject(sino, angles, fbp=False, method="exact", tol=1e-12):
    """Back-projection A^T y, src/backward.cpp:43-67 (+ ramp when fbp).

    Re(NUFFT1(fftshift(FFT(ifftshift(y))) [* ramp]))/D^2; sino [S, P, D] -> [S, D, D].
    """
    sino = np.asarray(sino, dtype=np.float64)
    S, P, D = sino.shape
    assert P == len(angles)
    c = np.fft.ifftshift(sino.astype(np.complex128), axes=-1)
    c = _fft(c, axis=-1)
    c = np.fft.fftshift(c, axes=-1)
    if fbp:
        c = c * ramp_filter(D)[None, None, :]
    x, y = polar_grid(P, D, angles)
    f = nufft_type1(c.reshape(S, P * D), x, y, D, method, tol)
    return f.real / float(D * D)


# --------------------------------------------------------------------------
# Toeplitz operator (PSF)
# --------------------------------------------------------------------------
def psf_kernel(n, angles, method="exact", tol=1e-12):
    """PSF = Re(NUFFT1(ones; (2n-1)^2 modes)), src/toeplitz.h:51-73.

    Returns the real [2n-1, 2n-1] array; index a <-> offset a - (n-1).
    """
    P = len(angles)
    m1 = 2 * n - 1
    x, y = polar_grid(P, n, angles)
    ones = np.ones((1, P * n), dtype=np.complex128)
    if method == "exact":
        f = nudft_type1(ones, x, y, m1)
    else:  # ES grid sized for the (odd) mode count, extracted the same way
        f = es_type1(ones, x, y, m1, tol)
    return f[0].real


class PsfSpectrum:
    """A point-spread function with its 2-D real FFT computed once, accepted
    wherever `psf` is (toeplitz_apply, gradient2, function_value2, ...) so a
    long solve does not transform the (2N-1)^2 PSF on every product."""

    def __init__(self, psf):
        self.psf = np.asarray(psf, dtype=np.float64)
        self.shape = self.psf.shape
        self.spec = _rfft2(self.psf)


def toeplitz_apply(x, psf):
    """H x = crop_{N-1}(IFFT2(FFT2(pad x) * FFT2(psf))) / N^3, src/toeplitz.h:107-132.

    The reference pads x (RIGHT, top-left) to (2N-1)^2, crops with offset
    N-1 (src/gpu/padding.cu:109-205) and divides by N^3 (2N-1)^2 where the
    (2N-1)^2 undoes cuFFT's unnormalised C2R; numpy's irfft2 already
    normalises, leaving 1/N^3.  Equivalent to the linear convolution
    (Hx)[k] = sum_m x[m] psf[k - m + (N-1)] / N^3.
    """
    x = np.asarray(x, dtype=np.float64)
    S, N, _ = x.shape
    m1 = psf.shape[0]
    assert m1 == 2 * N - 1
    xp = np.zeros((S, m1, m1))
    xp[:, :N, :N] = x
    pspec = psf.spec if isinstance(psf, PsfSpectrum) else _rfft2(psf)
    spec = _rfft2(xp) * pspec[None]
    out = _irfft2(spec, (m1, m1))
    return out[:, N - 1:2 * N - 1, N - 1:2 * N - 1] / float(N) ** 3


def gradient2(x, sinoT, psf):
    """Toeplitz data gradient H x - A^T y, src/gradient2.cpp:37-68 (line 62)."""
    return toeplitz_apply(x, psf) - np.asarray(sinoT, dtype=np.float64)


def gradient(x, sinoT, angles, method="exact", tol=1e-12):
    """NUFFT-pair gradient Re(NUFFT1(NUFFT2(x)))/N^3 - A^T y, src/gradient.cpp:35-71."""
    x = np.asarray(x, dtype=np.float64)
    S, N, _ = x.shape
    P = len(angles)
    gx, gy = polar_grid(P, N, angles)
    c = nufft_type2(x.astype(np.complex128), gx, gy, method, tol)
    f = nufft_type1(c, gx, gy, N, method, tol)
    return f.real / float(N) ** 3 - np.asarray(sinoT, dtype=np.float64)


def function_value2(x, sinoT, psf, sino_sq):
    """sum(x . Hx - 2 x . A^T y) + ||y||^2, src/error2.cpp:41-94."""
    x = np.asarray(x, dtype=np.float64)
    hx = toeplitz_apply(x, psf)
    return float(sino_sq + np.sum(x * hx) - 2.0 * np.sum(x * sinoT))


class ToeplitzCache:
    """gradient2 and function_value2 for one PSF, remembering H v for the last
    two arrays seen (by identity).  Optimizer::run2 asks for the gradient at y
    and then the objective at the new point and at the same y, and once more
    at the accepted point (src/optimize.h:113-150), so a long FP64 solve
    needs two Toeplitz products per attempt instead of four.  Same formulas
    and results as the functions above."""

    def __init__(self, psf):
        self.spec = psf if isinstance(psf, PsfSpectrum) else PsfSpectrum(psf)
        self._seen = []

    def hx(self, v):
        for a, h in self._seen:
            if a is v:
                return h
        h = toeplitz_apply(v, self.spec)
        self._seen = (self._seen + [(v, h)])[-2:]
        return h

    def gradient2(self, x, sinoT):
        return self.hx(x) - np.asarray(sinoT, dtype=np.float64)

    def function_value2(self, x, sinoT, sino_sq):
        x64 = np.asarray(x, dtype=np.float64)
        return float(sino_sq + np.sum(x64 * self.hx(x)) - 2.0 * np.sum(x64 * sinoT))


def function_value(x, sino, angles, method="exact", tol=1e-12):
    """||A x - y||^2, src/error.cpp:36-88."""
    r = project(x, angles, method, tol) - np.asarray(sino, dtype=np.float64)
    return float(np.sum(r * r))


# --------------------------------------------------------------------------
# qGGMRF prior
# --------------------------------------------------------------------------
def d_pot_func(delta, p, sigma):
    """rho'(delta), src/gpu/potential_function.cuh:90-108 (q = 2, c = MRF_C)."""
    delta = np.asarray(delta, dtype=np.float64)
    ad = np.abs(delta)
    sq = sigma ** MRF_Q
    sqp = sigma ** (MRF_Q - p)
    with np.errstate(divide="ignore", invalid="ignore"):
        t1 = ad ** (MRF_Q - p) / sqp
        t2 = ad ** (MRF_Q - 1.0)
        t3 = MRF_C + t1
        v = (t2 / (t3 * sq)) * (MRF_Q - ((MRF_Q - p) * t1) / t3)
    return np.where(delta > 0, v, np.where(delta < 0, -v, 0.0))


def qggmrf_grad(x, sigma, p=1.2, scale=1.0, use_core=True):
    """sum_{26 n} w_n rho'(x_v - x_n) with clamp-to-edge boundaries.

    src/gpu/cuTV2.cu:33-76 (kernel), src/gpu/dev_memory.cuh:88-94 (clamp),
    src/tv_update.cpp:76-106 (driver; the halo slices make the clamp global).
    Returns the prior gradient alone (the reference adds it into g in place).
    """
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    S, R, C = x.shape
    if use_core:
        g = np.zeros_like(x)
        w = np.ascontiguousarray(QGGMRF_WEIGHTS)
        _core().orc_qggmrf(S, R, C, _dptr(x), _dptr(g), float(sigma), float(p),
                           MRF_C, _dptr(w), float(scale))
        return g
    xp = np.pad(x, 1, mode="edge")
    g = np.zeros_like(x)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                wgt = QGGMRF_WEIGHTS[dz, dy, dx]
                if wgt == 0.0:
                    continue
                nb = xp[dz:dz + S, dy:dy + R, dx:dx + C]
                g += wgt * d_pot_func(x - nb, p, sigma)
    return scale * g


# --------------------------------------------------------------------------
# derivatives of the prior and the objective beyond the gradient (for the
# differentiable forms; the reference only evaluates the gradient).  The
# clamped stencil of qggmrf_grad is the exact gradient of
#   U(x) = 1/2 sum_v sum_{26 d} w_d rho(x_v - x_c(v+d)),
#   rho(delta) = u^2 / (c + u^(2-p)),  u = |delta| / sigma,
# the potential of src/gpu/potential_function.cuh:31-88 (q = 2).
# --------------------------------------------------------------------------
def pot_func(delta, p, sigma):
    """rho(delta) (src/gpu/potential_function.cuh:56-70 with q = 2)."""
    u2 = (np.asarray(delta, dtype=np.float64) / sigma) ** 2
    t = u2 ** ((MRF_Q - p) / 2.0)
    return u2 / (MRF_C + t)


def d2_pot_func(delta, p, sigma):
    """rho''(delta) = (A + (2 - p) t A'(t)) / sigma^2, A = (2c + p t)/(c + t)^2,
    A' = ((p - 4) c - p t)/(c + t)^3, t = (|delta|/sigma)^(2-p)."""
    d = np.abs(np.asarray(delta, dtype=np.float64))
    t = (d / sigma) ** (MRF_Q - p)
    A = (2.0 * MRF_C + p * t) / (MRF_C + t) ** 2
    Ap = ((p - 4.0) * MRF_C - p * t) / (MRF_C + t) ** 3
    return (A + (MRF_Q - p) * t * Ap) / sigma ** 2


def _neighbours(x):
    """(weight, clamped neighbour array) for the 26 offsets."""
    S, R, C = x.shape
    xp = np.pad(x, 1, mode="edge")
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                w = QGGMRF_WEIGHTS[dz, dy, dx]
                if w != 0.0:
                    yield w, xp[dz:dz + S, dy:dy + R, dx:dx + C]


def qggmrf_value(x, sigma, p=1.2):
    """(U(x), dU/dsigma); d rho / d sigma = -delta rho'(delta) / sigma."""
    x = np.asarray(x, dtype=np.float64)
    u = 0.0
    du = 0.0
    for w, nb in _neighbours(x):
        d = x - nb
        u += w * float(np.sum(pot_func(d, p, sigma)))
        du += w * float(np.sum(-d * d_pot_func(d, p, sigma) / sigma))
    return 0.5 * u, 0.5 * du


def qggmrf_hvp(x, v, sigma, p=1.2, scale=1.0):
    """(scale Hess U(x) v, v.grad U(x), v.dgrad U/dsigma);
    d rho'/d sigma = -(delta rho''(delta) + rho'(delta)) / sigma."""
    x = np.asarray(x, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    hv = np.zeros_like(x)
    g = np.zeros_like(x)
    gs = np.zeros_like(x)
    vnb = list(_neighbours(v))
    for (w, nb), (_, vn) in zip(_neighbours(x), vnb):
        d = x - nb
        d1 = d_pot_func(d, p, sigma)
        d2 = d2_pot_func(d, p, sigma)
        hv += w * d2 * (v - vn)
        g += w * d1
        gs += w * (-(d * d2 + d1) / sigma)
    return scale * hv, float(np.sum(v * g)), float(np.sum(v * gs))


def mbir_objective(x, sinoT, psf, sino_sq, sigma, p=1.2, beta=1.0):
    """F(x) = 1/2 ||A x - y||^2 + beta U(x), with ||A x - y||^2 =
    x.Hx - 2 x.A^T y + ||y||^2 (src/error2.cpp:41-63); its gradient is
    gradient2 + beta * qggmrf_grad (src/mbir2.cpp:122-129)."""
    return 0.5 * function_value2(x, sinoT, psf, sino_sq) + beta * qggmrf_value(x, sigma, p)[0]


def unrolled_mbir(x0, sinoT, psf, num_iters, step, beta, sigma, p=1.2, nesterov=False):
    """K fixed-step iterations x <- x - step (H x - A^T y + beta grad U(x)).

    Without nesterov this is Optimizer::run2's accepted-step path
    (src/optimize.h:117-146: after an accepted step x = sol, so the momentum
    term vanishes and the update is a gradient step).  With nesterov the
    FISTA extrapolation y = s + (t_k - 1)/t_{k+1} (s - s_prev) is applied."""
    s = np.asarray(x0, dtype=np.float64).copy()
    prev = s.copy()
    t = 1.0
    for _ in range(num_iters):
        if nesterov:
            tn = 0.5 * (1.0 + math.sqrt(1.0 + 4.0 * t * t))
            y = s + ((t - 1.0) / tn) * (s - prev)
            t = tn
        else:
            y = s
        g = gradient2(y, sinoT, psf) + qggmrf_grad(y, sigma, p, beta)
        prev = s
        s = y - step * g
    return s


def add_total_var2(x, g, sigma, p=1.2, scale=1.0):
    """In-place g += prior gradient (src/tv_update.cpp:76-106)."""
    g += qggmrf_grad(x, sigma, p, scale)
    return g


# --------------------------------------------------------------------------
# pre/post-processing
# --------------------------------------------------------------------------
def _cround(v):
    """std::round: halves away from zero."""
    return int(math.copysign(math.floor(abs(v) + 0.5), v))


def preproc_params(ncols, center):
    """npad and roll offset of src/preproc.cpp:79-85."""
    cen = _cround(float(center))
    cen_offset = (ncols + 1) // 2 - cen
    npad = int(0.42 * ncols) // 2
    if abs(cen_offset) > npad:
        npad = abs(cen_offset)
    return npad, cen_offset


def preproc(sino, center):
    """Detector pad (SYMMETRIC, npad per side) and roll, src/preproc.cpp:38-108."""
    sino = np.asarray(sino)
    S, P, D = sino.shape
    npad, off = preproc_params(D, center)
    out = np.zeros((S, P, D + 2 * npad), dtype=sino.dtype)
    out[:, :, npad:npad + D] = sino          # pad1d SYMMETRIC, shift = npad
    return np.roll(out, -off, axis=-1)       # roll_kernel: out[z] = in[z + off]


def postproc(soln, npixels):
    """Crop back to npixels, src/postproc.cpp:37-102."""
    soln = np.asarray(soln)
    S, R, C = soln.shape
    npad = (C - npixels) // 2
    return soln[:, npad:R - npad, npad:C - npad].copy()


def pad2d_symmetric(x, npad):
    """pad2d(.., SYMMETRIC): grow by npad, shift npad//2, src/padding.cpp:69-91."""
    x = np.asarray(x)
    S, R, C = x.shape
    sh = npad // 2
    out = np.zeros((S, R + npad, C + npad), dtype=x.dtype)
    out[:, sh:sh + R, sh:sh + C] = x
    return out


# --------------------------------------------------------------------------
# solver
# --------------------------------------------------------------------------
@dataclass
class Run2Record:
    iters: list = field(default_factory=list)     # (iter, error, xerr) per iteration
    attempts: int = 0


def run2(sol, num_iters, step_size, grad_fn, err_fn, record: Run2Record | None = None):
    """Nesterov with backtracking, Optimizer::run2 (src/optimize.h:96-154).

    Reproduced as written: beta = tnew (1/t - 1) with the current tnew;
    after acceptance x = sol, so the next y equals sol; a rejected attempt
    retries from the overwritten sol; step reset to step0 on acceptance;
    the test is sqrt f(sol) > sqrt f(y) + 0.5 step ||g||^2.  tol/xtol unused.
    """
    sol = np.array(sol, dtype=np.float64)
    x = sol.copy()
    t = 1.0
    tnew = 1.0
    step0 = step_size
    xerr = float(sol.size)
    for it in range(num_iters):
        while True:
            beta = tnew * (1.0 / t - 1.0)
            tnew = 0.5 * (math.sqrt(t ** 4 + 4.0 * t ** 2) - t ** 2)
            y = sol + (sol - x) * beta
            g = grad_fn(y)
            sol = y - g * step_size
            fx = err_fn(sol)
            fy = err_fn(y)
            gy = 0.5 * step_size * float(np.sum(g * g))
            if record is not None:
                record.attempts += 1
            if fx > fy + gy:
                step_size *= 0.9
            else:
                step_size = step0
                t = tnew
                xerr = float(np.sum((sol - x) ** 2))
                x = sol.copy()
                break
        e = err_fn(sol)
        if record is not None:
            record.iters.append((it, e, math.sqrt(xerr)))
    return sol


def lipschitz_step(psf, n):
    """step = min(1 / max(A^T A 1), 1), src/mbir2.cpp:100-112.

    The reference evaluates A^T A 1 with the NUFFT-pair gradient of ones; that
    equals the Toeplitz product H 1 (src/gradient.cpp:61-65 vs
    src/toeplitz.h:107-132).  add_tv_hessian (src/gpu/tv_hessian.cu:53-65)
    writes to a discarded device copy, so it contributes nothing.
    """
    h1 = toeplitz_apply(np.ones((1, n, n)), psf)
    L = float(h1.max())
    step = 1.0 / L
    return min(step, 1.0), L


def mbir2(sino, angles, center, num_iters, sigma, tol=1e-4, xtol=1e-4,
          method="exact", nufft_tol=1e-12, p=1.2, record: Run2Record | None = None,
          guess=None, beta=1.0):
    """Full MBIR, tomocam::mbir2 (src/mbir2.cpp:41-145).

    beta scales the prior gradient; the reference has no such factor and
    corresponds to beta = 1.
    """
    sino = np.asarray(sino, dtype=np.float64)
    if sino.ndim == 2:
        sino = sino[None]
    maxv = float(sino.max())
    if maxv == 0.0:
        raise RuntimeError("sinogram has ZERO max value")
    sino2 = sino / maxv
    if guess is None:
        x0 = backproject(sino2, angles, fbp=True, method=method, tol=nufft_tol)
    else:
        x0 = np.asarray(guess, dtype=np.float64)
    nrays = sino.shape[2]
    sino2 = preproc(sino2, center)
    npad = sino2.shape[2] - x0.shape[2]
    x0 = pad2d_symmetric(x0, npad)
    n = sino2.shape[2]
    sinoT = backproject(sino2, angles, fbp=False, method=method, tol=nufft_tol)
    sino_norm = float(np.sum(sino2 * sino2))
    psf = psf_kernel(n, angles, method, nufft_tol)
    step, _ = lipschitz_step(psf, n)

    def grad_fn(v):
        g = gradient2(v, sinoT, psf)
        return add_total_var2(v, g, sigma, p, beta)

    def err_fn(v):
        return math.sqrt(function_value2(v, sinoT, psf, sino_norm))

    rec = run2(x0, num_iters, step, grad_fn, err_fn, record)
    return postproc(rec, nrays)


# --------------------------------------------------------------------------
# synthetic inputs (seeded)
# --------------------------------------------------------------------------
def ellipse_phantom(n, n_ellipses=10, seed=0, lo=0.1, hi=1.0):
    """Seeded random-ellipse phantom on an n x n grid (float64)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    xx = (xx - (n - 1) / 2) / (n / 2)
    yy = (yy - (n - 1) / 2) / (n / 2)
    img = np.zeros((n, n))
    for _ in range(n_ellipses):
        cx, cy = rng.uniform(-0.5, 0.5, 2)
        ax, ay = rng.uniform(0.08, 0.4, 2)
        th = rng.uniform(0, np.pi)
        rho = rng.uniform(lo, hi)
        xr = (xx - cx) * np.cos(th) + (yy - cy) * np.sin(th)
        yr = -(xx - cx) * np.sin(th) + (yy - cy) * np.cos(th)
        img[(xr / ax) ** 2 + (yr / ay) ** 2 <= 1.0] += rho
    return img


def uniform_angles(nproj):
    """nproj angles uniform on [0, pi)."""
    return np.arange(nproj, dtype=np.float64) * (np.pi / nproj)
