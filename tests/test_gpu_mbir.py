"""MBIR solver parity through the C ABI against the FP64 oracle.

Reconstructions are held to 1e-4 relative L2 error against the FP64 oracle.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import phantom_stack, rel_l2

pytestmark = pytest.mark.gpu

TOL_RECON = 1e-4


def _setup(n=32, P=40, S=3, seed=0):
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    img = phantom_stack(S, n, seed=seed).astype(np.float64)
    sino = O.project(img, a64)
    sino = sino + 0.01 * sino.max() * np.random.default_rng(seed).standard_normal(sino.shape)
    aty = O.backproject(sino, a64)
    x0 = O.backproject(sino, a64, fbp=True)
    return ang, a64, sino, aty, x0


def _oracle_run(a64, n, sino, aty, x0, iters, sigma, p, step, weight=1.0):
    psf = O.psf_kernel(n, a64)
    sino_sq = float(np.sum(sino ** 2))
    if step <= 0:
        step, _ = O.lipschitz_step(psf, n)

    def grad_fn(v):
        g = O.gradient2(v, aty, psf)
        return g + O.qggmrf_grad(v, sigma, p, weight)

    def err_fn(v):
        return math.sqrt(O.function_value2(v, aty, psf, sino_sq))

    rec = O.Run2Record()
    x = O.run2(x0, iters, step, grad_fn, err_fn, rec)
    return x, rec, sino_sq


@pytest.mark.parametrize("use_graph", [True, False])
def test_solve_matches_oracle(use_graph):
    import torch
    from tomocam_b200.plan import Plan
    n = 32
    ang, a64, sino, aty, x0 = _setup(n)
    sigma, p, iters = 5.0, 1.2, 8
    ref, rec, sino_sq = _oracle_run(a64, n, sino, aty, x0, iters, sigma, p, 0.0)
    with Plan(n, ang) as pl:
        x, hist = pl.mbir_solve(torch.from_numpy(aty.astype(np.float32)).cuda(), sino_sq,
                                torch.from_numpy(x0.astype(np.float32)).cuda(), iters, sigma, p,
                                use_graph=use_graph)
    assert rel_l2(x.cpu().numpy(), ref) < TOL_RECON
    err_ref = np.array([e for _, e, _ in rec.iters])
    assert rel_l2(hist[:, 0], err_ref) < TOL_RECON


def test_backtracking_matches_oracle():
    """The retry path of run2 (rejected attempts, momentum from the overwritten sol).

    run2 rejects only when sqrt f(new) > sqrt f(y) + step/2 |g|^2, which needs
    a small gradient norm: the data are scaled by 1e-4 and the step is 2.5/L.
    """
    import torch
    from tomocam_b200.plan import Plan
    n = 32
    ang, a64, sino, aty, x0 = _setup(n, S=2, seed=3)
    sino, aty, x0 = sino * 1e-4, aty * 1e-4, x0 * 1e-4
    psf = O.psf_kernel(n, a64)
    step0, _ = O.lipschitz_step(psf, n)
    step = 2.5 * step0
    ref, rec, sino_sq = _oracle_run(a64, n, sino, aty, x0, 5, 1.0, 1.2, step, weight=1e-3)
    assert rec.attempts > 10  # the oracle did backtrack
    with Plan(n, ang) as pl:
        x, hist = pl.mbir_solve(torch.from_numpy(aty.astype(np.float32)).cuda(), sino_sq,
                                torch.from_numpy(x0.astype(np.float32)).cuda(), 5, 1.0, 1.2,
                                prior_weight=1e-3, step=step)
    assert rel_l2(x.cpu().numpy(), ref) < TOL_RECON
    err_ref = np.array([e for _, e, _ in rec.iters])
    assert rel_l2(hist[:, 0], err_ref) < TOL_RECON


def test_graph_and_plain_agree():
    import torch
    from tomocam_b200.plan import Plan
    n = 48
    ang, a64, sino, aty, x0 = _setup(n, P=30, S=4, seed=5)
    sino_sq = float(np.sum(sino ** 2))
    with Plan(n, ang) as pl:
        args = (torch.from_numpy(aty.astype(np.float32)).cuda(), sino_sq,
                torch.from_numpy(x0.astype(np.float32)).cuda(), 6, 2.0, 1.2)
        xg, hg = pl.mbir_solve(*args, use_graph=True)
        xp, hp = pl.mbir_solve(*args, use_graph=False)
    assert torch.equal(xg, xp)
    assert np.array_equal(hg, hp)


def test_mbir_host_matches_golden():
    """cTomocam.mbir (tomocam::mbir2 semantics) against the committed FP64 run."""
    from tests.golden import load
    import tomocam_b200 as tomocam
    g = load("mbir_n24")
    out = tomocam.MBIR(g["sino"], g["angles"], float(g["center"]), int(g["num_iters"]),
                       smoothness=1.0 / float(g["sigma"]))
    assert out.shape == g["out"].shape
    assert rel_l2(out, g["out"]) < TOL_RECON


def test_mbir_host_matches_oracle_live():
    import tomocam_b200 as tomocam
    D, P = 40, 36
    ang = O.uniform_angles(P).astype(np.float32)
    img = phantom_stack(2, D, seed=9).astype(np.float64)
    sino = O.project(img, ang.astype(np.float64)).astype(np.float32)
    ref = O.mbir2(sino, ang.astype(np.float64), 20.3, 5, sigma=10.0)
    out = tomocam.MBIR(sino, ang, 20.3, 5, smoothness=0.1)
    assert rel_l2(out, ref) < TOL_RECON


def test_mbir_zero_sinogram_raises():
    import tomocam_b200 as tomocam
    with pytest.raises(RuntimeError, match="ZERO max"):
        tomocam.MBIR(np.zeros((1, 10, 16), np.float32), O.uniform_angles(10).astype(np.float32),
                     8.0, 2)



def _single_slice_256():
    ang = O.uniform_angles(180).astype(np.float32).astype(np.float64)
    img = O.ellipse_phantom(256, 10, seed=0)[None]
    sino = O.project(img, ang, "es", 1e-12)
    sino = sino + 0.01 * sino.max() * np.random.default_rng(0).standard_normal(sino.shape)
    return ang, sino.astype(np.float32).astype(np.float64)


def test_mbir_single_slice_256():
    """One 256 x 256 slice of ten random ellipses, 180 angles, 256 detector
    pixels centred at 128, 1 % Gaussian noise; qGGMRF p = 1.2, smoothness
    0.05 (sigma = 20), prior weight 0.5; 20 iterations through the
    reference-facing MBIR call against the FP64 oracle's mbir2
    (exponential-of-semicircle NUFFT at 1e-12)."""
    import tomocam_b200 as tomocam
    ang, sino = _single_slice_256()
    ref = O.mbir2(sino, ang, 128.0, 20, sigma=20.0, method="es", nufft_tol=1e-12, beta=0.5)
    out = tomocam.MBIR(sino.astype(np.float32), ang.astype(np.float32), 128.0, 20,
                       smoothness=0.05, beta=0.5)
    assert out.shape == (1, 256, 256)
    assert rel_l2(out, ref) < TOL_RECON


def test_mbir_single_slice_256_sharp_prior():
    """The same slice with sigma = 0.05 itself: the step 1/max(H 1) ignores
    the prior's curvature (~1/sigma^2), so run2 is unstable here (the
    objective rises in the first iterations) and the FP64 result moves by
    3e-6, 3e-5 and 6e-4 under a 6e-8 perturbation of the input after 1, 2
    and 3 iterations.  The first iteration, before the instability has
    grown, is held to the reconstruction tolerance."""
    import tomocam_b200 as tomocam
    ang, sino = _single_slice_256()
    ref = O.mbir2(sino, ang, 128.0, 1, sigma=0.05, method="es", nufft_tol=1e-12, beta=0.5)
    out = tomocam.MBIR(sino.astype(np.float32), ang.astype(np.float32), 128.0, 1,
                       smoothness=1.0 / 0.05, beta=0.5)
    assert rel_l2(out, ref) < TOL_RECON


def test_graph_reused_and_recaptured():
    """The plan keeps the instantiated solver graph for the next solve with the
    same captured arguments; a changed prior parameter (captured by value) or
    a different A^T y buffer (captured address) must capture a new one.  Every
    graph solve equals the host-driven solve of the same inputs."""
    import torch
    from tomocam_b200.plan import Plan
    n = 40
    ang, a64, sino, aty, x0 = _setup(n, P=30, S=3, seed=8)
    sino_sq = float(np.sum(sino ** 2))
    aty_d = torch.from_numpy(aty.astype(np.float32)).cuda()
    x0_d = torch.from_numpy(x0.astype(np.float32)).cuda()
    with Plan(n, ang) as pl:
        def pair(a, sigma):
            xg, hg = pl.mbir_solve(a, sino_sq, x0_d.clone(), 5, sigma, 1.2, use_graph=True)
            xp, hp = pl.mbir_solve(a, sino_sq, x0_d.clone(), 5, sigma, 1.2, use_graph=False)
            assert torch.equal(xg, xp)
            assert np.array_equal(hg, hp)
            return xg
        first = pair(aty_d, 2.0)
        again = pair(aty_d, 2.0)                 # reused graph
        assert torch.equal(first, again)
        other_sigma = pair(aty_d, 7.0)           # prior parameters changed
        assert not torch.equal(first, other_sigma)
        aty2 = (aty_d * 0.5).contiguous()
        other_aty = pair(aty2, 2.0)              # another A^T y buffer
        assert not torch.equal(first, other_aty)
