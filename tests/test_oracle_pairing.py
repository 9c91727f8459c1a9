"""The two-slices-per-line scheme of the register-FFT NUFFT path, restated in
FP64 numpy on the oracle's exact non-uniform DFT (CPU).

The CUDA path carries slices a and b as the real and imaginary parts of one
complex line.  Each slice comes back exactly only if its transform is real,
i.e. if the point values it feeds or receives are Hermitian-symmetric over
the polar point set.  The radii s (j - D//2) are symmetric for odd D; for
even D the sample j = 0 (radius -s D/2) has no partner, so the CUDA path
adds one mirror point at +s D/2 per angle and splits the unpaired sample:
radon replaces the j = 0 value by the mean of the values at -+s D/2,
back-projection puts half of the (real) j = 0 detector coefficient on the
point and half on its mirror, the NUFFT gradient halves both interpolated
values.  These tests show, at sizes the exact DFT finishes in milliseconds,
that the restated scheme gives each slice's unpaired result (oracle.project,
oracle.backproject, oracle.gradient) to FP64 rounding.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _mirror(P, D, angles):
    s = 2.0 * np.pi / (D - 1)
    rm = s * (D - D // 2)
    ang = np.asarray(angles, dtype=np.float64)
    return rm * np.cos(ang), rm * np.sin(ang)


def _pair(rng, shape):
    return rng.standard_normal(shape), rng.standard_normal(shape)


def paired_project(xa, xb, angles):
    N = xa.shape[-1]
    P, D = len(angles), N
    gx, gy = O.polar_grid(P, D, angles)
    z = (xa + 1j * xb)[None]
    c = O.nufft_type2(z, gx, gy).reshape(P, D)
    if D % 2 == 0:
        mx, my = _mirror(P, D, angles)
        m = O.nufft_type2(z, mx, my).reshape(P)
        c[:, 0] = 0.5 * (c[:, 0] + m)
    c = np.fft.ifftshift(c, axes=-1)
    c = O._fft(c, axis=-1, inverse=True) * D
    y = np.fft.fftshift(c, axes=-1) / float(N * N)
    return y.real, y.imag


def paired_backproject(ya, yb, angles, fbp):
    P, D = ya.shape
    gx, gy = O.polar_grid(P, D, angles)
    c = np.fft.ifftshift((ya + 1j * yb).astype(np.complex128), axes=-1)
    c = O._fft(c, axis=-1)
    c = np.fft.fftshift(c, axes=-1)
    if fbp:
        c = c * O.ramp_filter(D)[None, :]
    xs, ys, cs = gx.reshape(-1), gy.reshape(-1), c.reshape(-1)
    if D % 2 == 0:
        mx, my = _mirror(P, D, angles)
        half = 0.5 * c[:, 0]
        cs = c.copy()
        cs[:, 0] = half
        xs, ys = np.concatenate([xs, mx]), np.concatenate([ys, my])
        cs = np.concatenate([cs.reshape(-1), half])
    f = O.nufft_type1(cs[None], xs, ys, D)[0] / float(D * D)
    return f.real, f.imag


def paired_gradient(xa, xb, angles):
    N = xa.shape[-1]
    P = len(angles)
    gx, gy = O.polar_grid(P, N, angles)
    xs, ys = gx.reshape(-1), gy.reshape(-1)
    if N % 2 == 0:
        mx, my = _mirror(P, N, angles)
        xs, ys = np.concatenate([xs, mx]), np.concatenate([ys, my])
    c = O.nufft_type2((xa + 1j * xb)[None], xs, ys)[0]
    if N % 2 == 0:
        j0 = np.arange(P) * N
        c[j0] *= 0.5
        c[P * N:] *= 0.5
    f = O.nufft_type1(c[None], xs, ys, N)[0] / float(N) ** 3
    return f.real, f.imag


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("N", [16, 15, 24])
def test_paired_radon_gives_each_slice(N):
    rng = np.random.default_rng(N)
    ang = O.uniform_angles(7)
    xa, xb = _pair(rng, (N, N))
    ya, yb = paired_project(xa, xb, ang)
    assert _rel(ya, O.project(xa[None], ang)[0]) < 1e-12
    assert _rel(yb, O.project(xb[None], ang)[0]) < 1e-12


@pytest.mark.parametrize("N", [16, 15, 24])
@pytest.mark.parametrize("fbp", [False, True])
def test_paired_backprojection_gives_each_slice(N, fbp):
    rng = np.random.default_rng(N + 100)
    ang = O.uniform_angles(7)
    ya, yb = _pair(rng, (7, N))
    fa, fb = paired_backproject(ya, yb, ang, fbp)
    assert _rel(fa, O.backproject(ya[None], ang, fbp=fbp)[0]) < 1e-12
    assert _rel(fb, O.backproject(yb[None], ang, fbp=fbp)[0]) < 1e-12


@pytest.mark.parametrize("N", [16, 15])
def test_paired_nufft_gradient_gives_each_slice(N):
    rng = np.random.default_rng(N + 200)
    ang = O.uniform_angles(7)
    xa, xb = _pair(rng, (N, N))
    ga, gb = paired_gradient(xa, xb, ang)
    zero = np.zeros((1, N, N))
    assert _rel(ga, O.gradient(xa[None], zero, ang)[0]) < 1e-12
    assert _rel(gb, O.gradient(xb[None], zero, ang)[0]) < 1e-12


def test_even_detector_needs_the_mirror_point():
    """Without the mirror point the unpaired j = 0 sample mixes the slices:
    for even D the plain paired radon differs from the unpaired one."""
    N = 16
    rng = np.random.default_rng(5)
    ang = O.uniform_angles(7)
    xa, xb = _pair(rng, (N, N))
    gx, gy = O.polar_grid(7, N, ang)
    c = O.nufft_type2((xa + 1j * xb)[None], gx, gy).reshape(7, N)
    c = np.fft.ifftshift(c, axes=-1)
    c = O._fft(c, axis=-1, inverse=True) * N
    y = np.fft.fftshift(c, axes=-1) / float(N * N)
    assert _rel(y.real, O.project(xa[None], ang)[0]) > 1e-6
