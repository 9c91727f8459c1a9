"""torch.autograd forms against the FP64 oracle: the radon adjoint, the MBIR
objective and its gradient (the reference's gradient2 + qGGMRF stencil), the
vector-Jacobian products of the gradient, and d/dbeta, d/dsigma of an
unrolled, checkpointed reconstruction against FP64 central differences."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2
from tests.test_oracle_diff import unrolled_loss_fd

pytestmark = pytest.mark.gpu

SIGMA, P_PRIOR, BETA = 0.05, 1.2, 0.5


@pytest.fixture(scope="module")
def setup():
    import torch
    from tomocam_b200.plan import Plan
    n, P, S = 64, 90, 2
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    img = np.stack([O.ellipse_phantom(n, 10, s) for s in range(S)])
    sino = O.project(img, a64)
    aty32 = O.backproject(sino, a64).astype(np.float32)
    psf = O.psf_kernel(n, a64)
    pl = Plan(n, ang, psf=False)
    pl.set_psf(psf)
    d = dict(n=n, ang=a64, img=img, sino=sino, aty=aty32.astype(np.float64), psf=psf,
             sino_sq=float(np.sum(sino ** 2)), plan=pl,
             aty_t=torch.from_numpy(aty32).cuda())
    yield d
    pl.close()


def _t(a, grad=False):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()
    return t.requires_grad_(grad)


def _p(v):
    import torch
    return torch.tensor(v, dtype=torch.float64, requires_grad=True)


def test_radon_backward_is_the_adjoint(setup):
    import torch
    from tomocam_b200.autograd import radon
    pl = setup["plan"]
    rng = np.random.default_rng(0)
    x = _t(rng.standard_normal((2, 64, 64)), grad=True)
    y = _t(rng.standard_normal((2, 90, 64)))
    ax = radon(x, pl)
    (ax * y).sum().backward()
    # the back-projection's spreading accumulates with atomics: compare to rounding
    assert rel_l2(x.grad.cpu().numpy(), pl.iradon(y).cpu().numpy()) < 1e-6
    lhs = float((ax.detach().double() * y.double()).sum())
    rhs = float((x.detach().double() * x.grad.double()).sum())
    assert abs(lhs - rhs) / (float(ax.detach().double().norm()) * float(y.double().norm())) < 1e-5


def test_objective_and_gradients_match_oracle(setup):
    from tomocam_b200.autograd import mbir_objective
    d = setup
    x64 = d["img"] + 0.05 * np.random.default_rng(1).standard_normal(d["img"].shape)
    x = _t(x64, grad=True)
    x64 = x.detach().cpu().numpy().astype(np.float64)
    beta, sigma = _p(BETA), _p(SIGMA)
    f = mbir_objective(x, d["plan"], d["aty_t"], d["sino_sq"], beta, sigma, P_PRIOR)
    f.backward()
    f_ref = O.mbir_objective(x64, d["aty"], d["psf"], d["sino_sq"], SIGMA, P_PRIOR, BETA)
    g_ref = O.gradient2(x64, d["aty"], d["psf"]) + O.qggmrf_grad(x64, SIGMA, P_PRIOR, BETA)
    u_ref, du_ref = O.qggmrf_value(x64, SIGMA, P_PRIOR)
    assert float(f) == pytest.approx(f_ref, rel=1e-5)
    assert rel_l2(x.grad.cpu().numpy(), g_ref) < 1e-5
    assert float(beta.grad) == pytest.approx(u_ref, rel=1e-5)
    assert float(sigma.grad) == pytest.approx(BETA * du_ref, rel=1e-5)


def test_objective_directional_derivative_on_device(setup):
    """forward and backward of the GPU objective agree (central differences
    of the FP32 objective along 5 random unit directions)."""
    import torch
    from tomocam_b200.autograd import mbir_objective
    d = setup
    x0 = d["img"] + 0.05 * np.random.default_rng(2).standard_normal(d["img"].shape)
    x = _t(x0, grad=True)
    mbir_objective(x, d["plan"], d["aty_t"], d["sino_sq"], BETA, SIGMA, P_PRIOR).backward()
    g = x.grad.double()
    rng = np.random.default_rng(3)
    h = 1e-2
    with torch.no_grad():
        for _ in range(5):
            v = _t(rng.standard_normal(x0.shape))
            v /= v.norm()
            f1 = mbir_objective(x + h * v, d["plan"], d["aty_t"], d["sino_sq"], BETA, SIGMA, P_PRIOR)
            f0 = mbir_objective(x - h * v, d["plan"], d["aty_t"], d["sino_sq"], BETA, SIGMA, P_PRIOR)
            fd = float(f1 - f0) / (2 * h)
            an = float((g * v.double()).sum())
            assert abs(fd - an) < 1e-2 * float(g.norm())


def test_gradient_vjp_matches_oracle(setup):
    """vector-Jacobian products of g = H x - A^T y + beta grad U."""
    from tomocam_b200.autograd import mbir_grad
    d = setup
    rng = np.random.default_rng(4)
    x64 = d["img"] + 0.05 * rng.standard_normal(d["img"].shape)
    v64 = rng.standard_normal(x64.shape)
    x = _t(x64, grad=True)
    aty = d["aty_t"].clone().requires_grad_(True)
    x64 = x.detach().cpu().numpy().astype(np.float64)
    v = _t(v64)
    v64 = v.cpu().numpy().astype(np.float64)
    beta, sigma = _p(BETA), _p(SIGMA)
    g = mbir_grad(x, d["plan"], aty, beta, sigma, P_PRIOR)
    (g * v).sum().backward()
    hv_ref = O.gradient2(v64, np.zeros_like(v64), d["psf"])
    hp_ref, vg_ref, vgs_ref = O.qggmrf_hvp(x64, v64, SIGMA, P_PRIOR, BETA)
    assert rel_l2(x.grad.cpu().numpy(), hv_ref + hp_ref) < 1e-4
    assert rel_l2(aty.grad.cpu().numpy(), -v64) == 0.0
    assert float(beta.grad) == pytest.approx(vg_ref, rel=1e-4)
    assert float(sigma.grad) == pytest.approx(BETA * vgs_ref, rel=1e-4)


@pytest.mark.parametrize("checkpoint_every", [1, 0])
def test_unrolled_parameter_gradients_match_fp64_fd(setup, checkpoint_every):
    """d/dbeta, d/dsigma of L = 1/2 ||x_K - x_true||^2 (K = 5) by backprop
    through the checkpointed unrolled reconstruction vs FP64 central
    differences of the oracle's unrolled reconstruction."""
    import torch
    from tomocam_b200.autograd import unrolled_mbir
    d = setup
    x0_64 = 0.9 * d["img"] + 0.02 * np.random.default_rng(5).standard_normal(d["img"].shape)
    x0 = _t(x0_64)
    x0_64 = x0.cpu().numpy().astype(np.float64)
    step, _ = O.lipschitz_step(d["psf"], d["n"])
    beta, sigma = _p(BETA), _p(SIGMA)
    xk = unrolled_mbir(x0, d["plan"], d["aty_t"], 5, 0.5 * step, beta, sigma, P_PRIOR,
                       checkpoint_every=checkpoint_every)
    xk_ref = O.unrolled_mbir(x0_64, d["aty"], d["psf"], 5, 0.5 * step, BETA, SIGMA, P_PRIOR)
    assert rel_l2(xk.detach().cpu().numpy(), xk_ref) < 1e-4
    loss = 0.5 * ((xk.double() - torch.from_numpy(d["img"]).cuda()) ** 2).sum()
    loss.backward()
    db_ref, ds_ref = unrolled_loss_fd(d, x0_64, BETA, SIGMA, 1e-7)
    assert float(beta.grad) == pytest.approx(db_ref, rel=2e-3)
    assert float(sigma.grad) == pytest.approx(ds_ref, rel=2e-3)


def test_unrolled_checkpointing_changes_nothing(setup):
    import torch
    from tomocam_b200.autograd import unrolled_mbir
    d = setup
    x0 = _t(0.9 * d["img"])
    grads = []
    for ck in (0, 1, 2):
        beta, sigma = _p(BETA), _p(SIGMA)
        xk = unrolled_mbir(x0, d["plan"], d["aty_t"], 4, 0.3, beta, sigma, P_PRIOR,
                           nesterov=True, checkpoint_every=ck)
        (xk.double() ** 2).sum().backward()
        grads.append((float(beta.grad), float(sigma.grad)))
    for gb, gs in grads[1:]:
        assert gb == pytest.approx(grads[0][0], rel=1e-6)
        assert gs == pytest.approx(grads[0][1], rel=1e-6)
