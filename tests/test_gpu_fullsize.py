"""Parity at the benchmark workloads' own in-plane sizes.

The oracle's exponential-of-semicircle NUFFT (FP64, tolerance 1e-10) is fast
enough at these sizes for a few slices, so the operators and a short solve
are checked directly against it at full size:

* operator pair: 1024 x 1024 phantoms on a 1536-pixel detector, 1500 angles;
* full-volume MBIR: 2048 x 2048 foam slices, 1969 angles, and the 2908-pixel
  grid that the detector padding of a 2048-pixel detector produces.

Operators are held to 1e-5 and reconstructions to 1e-4 relative L2 error.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_RECON = 1e-4
ES_TOL = 1e-10


def _ellipses_textured(S, n_img, n, seed):
    """n_img x n_img ellipse phantoms plus N(0, 0.01) texture, centred in n x n."""
    rng = np.random.default_rng(seed)
    out = np.zeros((S, n, n))
    o = (n - n_img) // 2
    for s in range(S):
        out[s, o:o + n_img, o:o + n_img] = (O.ellipse_phantom(n_img, 10, seed + s)
                                            + 0.01 * rng.standard_normal((n_img, n_img)))
    return out.astype(np.float32)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


@pytest.fixture(scope="module")
def pair_case():
    from tomocam_b200.plan import Plan
    n, P = 1536, 1500
    ang = O.uniform_angles(P).astype(np.float32)
    pl = Plan(n, ang)
    yield n, ang.astype(np.float64), pl
    pl.close()


def test_operator_pair_full_size(pair_case):
    n, a64, pl = pair_case
    x = _ellipses_textured(2, 1024, n, seed=1)
    y = pl.radon(_dev(x)).cpu().numpy()
    assert rel_l2(y, O.project(x.astype(np.float64), a64, "es", ES_TOL)) < TOL

    sino = np.random.default_rng(2).standard_normal((2, len(a64), n)).astype(np.float32)
    for ramp in (False, True):
        b = pl.iradon(_dev(sino), ramp=ramp).cpu().numpy()
        ref = O.backproject(sino.astype(np.float64), a64, fbp=ramp, method="es", tol=ES_TOL)
        assert rel_l2(b, ref) < TOL


def test_adjoint_full_size(pair_case):
    n, a64, pl = pair_case
    rng = np.random.default_rng(11)
    x = _dev(_ellipses_textured(4, 1024, n, seed=3))
    y = _dev(rng.standard_normal((4, len(a64), n)))
    ax = pl.radon(x).double()
    lhs = float((ax * y.double()).sum())
    rhs = float((x.double() * pl.iradon(y).double()).sum())
    assert abs(lhs - rhs) / (float(ax.norm()) * float(y.double().norm())) < 1e-5


def test_psf_and_toeplitz_full_size(pair_case):
    n, a64, pl = pair_case
    psf = O.psf_kernel(n, a64, "es", ES_TOL)
    assert rel_l2(pl.psf(), psf) < 1e-8
    x = _ellipses_textured(2, 1024, n, seed=5)
    aty = np.random.default_rng(6).standard_normal(x.shape).astype(np.float32)
    g, xhx, _ = pl.toeplitz_grad(_dev(x), _dev(aty), dots=True)
    hx = O.toeplitz_apply(x.astype(np.float64), psf)
    assert rel_l2(g.cpu().numpy(), hx - aty) < TOL
    assert abs(xhx - np.sum(x * hx)) / abs(np.sum(x * hx)) < TOL


def test_toeplitz_padded_grid_2908():
    """The grid of a 2048-pixel detector after the 0.42 x padding (2908
    pixels, FFT length 6144), with its own FP64 PSF for 1969 angles."""
    from tomocam_b200.plan import Plan
    n, P = 2908, 1969
    ang = O.uniform_angles(P).astype(np.float32)
    psf = O.psf_kernel(n, ang.astype(np.float64), "es", ES_TOL)
    x = np.random.default_rng(7).random((1, n, n)).astype(np.float32)
    aty = np.random.default_rng(8).standard_normal((1, n, n)).astype(np.float32)
    with Plan(n, ang) as pl:
        assert rel_l2(pl.psf(), psf) < 1e-8
        g = pl.toeplitz_grad(_dev(x), _dev(aty))
    hx = O.toeplitz_apply(x.astype(np.float64), psf)
    assert rel_l2(g.cpu().numpy(), hx - aty) < TOL


def test_solve_foam_slices_2048():
    """Four 2048 x 2048 slices of the seeded foam volume, 1969 angles,
    transmission noise at 1e4 counts, qGGMRF p = 1.2, sigma = 100; four
    graph-captured iterations against the oracle's run2."""
    import torch
    from tomocam_b200 import phantom
    from tomocam_b200.plan import Plan
    S, n, P, sigma, iters = 4, 2048, 1969, 100.0, 4
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    vol = phantom.foam_volume(S, n, 300, seed=0, device="cpu").numpy().astype(np.float64)
    sino = O.project(vol, a64, "es", ES_TOL)
    sino = phantom.transmission_noise(torch.from_numpy(sino.astype(np.float32)), 1e4, 3.0,
                                      seed=0).numpy().astype(np.float64)
    sino /= sino.max()
    sino = sino.astype(np.float32).astype(np.float64)
    aty = O.backproject(sino, a64, method="es", tol=ES_TOL).astype(np.float32).astype(np.float64)
    x0 = O.backproject(sino, a64, fbp=True, method="es", tol=ES_TOL)
    x0 = x0.astype(np.float32).astype(np.float64)
    sino_sq = float(np.sum(sino ** 2))

    psf = O.psf_kernel(n, a64, "es", ES_TOL)
    step, _ = O.lipschitz_step(psf, n)
    rec = O.Run2Record()
    ref = O.run2(x0, iters, step,
                 lambda v: O.gradient2(v, aty, psf) + O.qggmrf_grad(v, sigma, 1.2),
                 lambda v: math.sqrt(O.function_value2(v, aty, psf, sino_sq)), rec)

    with Plan(n, ang) as pl:
        x, hist = pl.mbir_solve(_dev(aty), sino_sq, _dev(x0), iters, sigma, 1.2, use_graph=True)
    assert rel_l2(x.cpu().numpy(), ref) < TOL_RECON
    err_ref = np.array([e for _, e, _ in rec.iters])
    assert rel_l2(hist[:, 0], err_ref) < TOL_RECON
