"""FP64 finite-difference checks of the derivative formulas the differentiable
forms use (prior potential, Hessian-vector product, sigma derivatives, the
MBIR objective and the unrolled reconstruction), on the CPU oracle."""
import numpy as np
import pytest

from oracle import oracle as O


def _rand(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


def test_prior_potential_gradient_is_the_clamped_stencil():
    """grad U equals the reference's clamp-to-edge 26-neighbour stencil,
    border voxels included (central differences, h = 1e-6)."""
    x = _rand((3, 4, 5), 0)
    sigma, p, h = 0.7, 1.2, 1e-6
    g = O.qggmrf_grad(x, sigma, p, use_core=False)
    fd = np.zeros_like(x)
    for idx in np.ndindex(x.shape):
        e = np.zeros_like(x)
        e[idx] = h
        fd[idx] = (O.qggmrf_value(x + e, sigma, p)[0] - O.qggmrf_value(x - e, sigma, p)[0]) / (2 * h)
    assert np.abs(g - fd).max() / np.abs(g).max() < 1e-7


def test_prior_hvp_and_sigma_terms():
    x, v = _rand((3, 5, 6), 1), _rand((3, 5, 6), 2)
    sigma, p, scale = 0.7, 1.2, 0.3
    hv, vg, vgs = O.qggmrf_hvp(x, v, sigma, p, scale)
    h = 1e-7
    g1 = O.qggmrf_grad(x + h * v, sigma, p, scale, use_core=False)
    g0 = O.qggmrf_grad(x - h * v, sigma, p, scale, use_core=False)
    assert np.abs(hv - (g1 - g0) / (2 * h)).max() / np.abs(hv).max() < 1e-6
    assert vg == pytest.approx(float(np.sum(v * O.qggmrf_grad(x, sigma, p, use_core=False))), rel=1e-12)
    hs = 1e-6
    dgs = (O.qggmrf_grad(x, sigma + hs, p, use_core=False) - O.qggmrf_grad(x, sigma - hs, p, use_core=False)) / (2 * hs)
    assert vgs == pytest.approx(float(np.sum(v * dgs)), rel=1e-7)
    du = (O.qggmrf_value(x, sigma + hs, p)[0] - O.qggmrf_value(x, sigma - hs, p)[0]) / (2 * hs)
    assert O.qggmrf_value(x, sigma, p)[1] == pytest.approx(du, rel=1e-7)


@pytest.fixture(scope="module")
def scan64():
    n, P, S = 64, 90, 2
    ang = O.uniform_angles(P)
    img = np.stack([O.ellipse_phantom(n, 10, s) for s in range(S)])
    sino = O.project(img, ang)
    aty = O.backproject(sino, ang)
    psf = O.psf_kernel(n, ang)
    return dict(n=n, ang=ang, img=img, sino=sino, aty=aty, psf=psf,
                sino_sq=float(np.sum(sino ** 2)))


def test_objective_gradient_fd(scan64):
    """dF/dx = H x - A^T y + beta grad U: central differences in FP64,
    h = 1e-6, 20 random directions, at 64^2 with 90 angles."""
    d = scan64
    sigma, p, beta = 0.05, 1.2, 0.5
    x = d["img"] + 0.05 * _rand(d["img"].shape, 3)
    g = O.gradient2(x, d["aty"], d["psf"]) + O.qggmrf_grad(x, sigma, p, beta)
    rng = np.random.default_rng(4)
    h = 1e-6
    worst = 0.0
    for _ in range(20):
        v = rng.standard_normal(x.shape)
        v /= np.linalg.norm(v)
        f1 = O.mbir_objective(x + h * v, d["aty"], d["psf"], d["sino_sq"], sigma, p, beta)
        f0 = O.mbir_objective(x - h * v, d["aty"], d["psf"], d["sino_sq"], sigma, p, beta)
        fd = (f1 - f0) / (2 * h)
        an = float(np.sum(g * v))
        worst = max(worst, abs(fd - an) / np.linalg.norm(g))
    assert worst < 1e-6


def unrolled_loss_fd(d, x0, beta, sigma, h, iters=5, frac=0.5):
    """Central differences of L = 1/2 ||x_K - x_true||^2 in beta and sigma."""
    step, _ = O.lipschitz_step(d["psf"], d["n"])

    def loss(b, s):
        xk = O.unrolled_mbir(x0, d["aty"], d["psf"], iters, frac * step, b, s)
        return 0.5 * float(np.sum((xk - d["img"]) ** 2))

    return ((loss(beta + h, sigma) - loss(beta - h, sigma)) / (2 * h),
            (loss(beta, sigma + h) - loss(beta, sigma - h)) / (2 * h))


def test_unrolled_parameter_derivatives_fd(scan64):
    """d/dbeta and d/dsigma of L = 1/2 ||x_K - x_true||^2 are well defined:
    central differences at h = 1e-6 and 1e-7 agree.  (rho'' has a
    |delta|^(2-p) cusp at delta = 0, so iterates whose neighbour differences
    cross zero make L only Hoelder-smooth there; a start near the solution
    keeps the differences away from zero.)"""
    d = scan64
    x0 = 0.9 * d["img"] + 0.02 * _rand(d["img"].shape, 5)
    a = unrolled_loss_fd(d, x0, 0.5, 0.05, 1e-6)
    b = unrolled_loss_fd(d, x0, 0.5, 0.05, 1e-7)
    for u, v in zip(a, b):
        assert abs(u - v) <= 1e-4 * abs(u)
