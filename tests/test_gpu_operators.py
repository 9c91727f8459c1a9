"""Operator parity through the C ABI against the FP64 oracle.

Operators are held to 1e-5 relative L2 error against the FP64 oracle (exact
non-uniform DFT at these sizes), the tolerance the MBIR path targets.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import phantom_stack, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5
CASES = [(32, 24), (33, 20), (48, 30), (64, 45)]


def _torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def plans():
    from tomocam_b200.plan import Plan
    out = {}
    for n, P in CASES:
        ang = O.uniform_angles(P).astype(np.float32)
        out[(n, P)] = (Plan(n, ang), ang)
    yield out
    for p, _ in out.values():
        p.close()


@pytest.mark.parametrize("case", CASES)
def test_radon(plans, case):
    torch = _torch()
    pl, ang = plans[case]
    n, P = case
    x = phantom_stack(3, n, seed=7)
    y = pl.radon(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = O.project(x.astype(np.float64), ang.astype(np.float64))
    assert y.shape == (3, P, n)
    assert rel_l2(y, ref) < TOL


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("ramp", [False, True])
def test_iradon(plans, case, ramp):
    torch = _torch()
    pl, ang = plans[case]
    n, P = case
    rng = np.random.default_rng(3)
    sino = rng.standard_normal((2, P, n)).astype(np.float32)
    x = pl.iradon(torch.from_numpy(sino).cuda(), ramp=ramp).cpu().numpy()
    ref = O.backproject(sino.astype(np.float64), ang.astype(np.float64), fbp=ramp)
    assert rel_l2(x, ref) < TOL


@pytest.mark.parametrize("case", CASES)
def test_adjoint(plans, case):
    torch = _torch()
    pl, _ = plans[case]
    n, P = case
    rng = np.random.default_rng(11)
    x = torch.from_numpy(rng.standard_normal((2, n, n)).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.standard_normal((2, P, n)).astype(np.float32)).cuda()
    ax = pl.radon(x)
    aty = pl.iradon(y)
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) / (float(ax.double().norm()) * float(y.double().norm())) < 1e-5


@pytest.mark.parametrize("case", CASES)
def test_psf_fp64(plans, case):
    pl, ang = plans[case]
    n, _ = case
    ref = O.psf_kernel(n, ang.astype(np.float64))
    assert rel_l2(pl.psf(), ref) < 1e-10


@pytest.mark.parametrize("case", CASES)
def test_toeplitz_grad(plans, case):
    torch = _torch()
    pl, ang = plans[case]
    n, _ = case
    rng = np.random.default_rng(5)
    for S in (1, 2, 3):
        x = phantom_stack(S, n, seed=2)
        aty = rng.standard_normal((S, n, n)).astype(np.float32)
        g, xhx, xaty = pl.toeplitz_grad(torch.from_numpy(x).cuda(), torch.from_numpy(aty).cuda(),
                                        dots=True)
        psf = O.psf_kernel(n, ang.astype(np.float64))
        hx = O.toeplitz_apply(x.astype(np.float64), psf)
        ref = hx - aty
        assert rel_l2(g.cpu().numpy(), ref) < TOL
        assert abs(xhx - np.sum(x * hx)) / abs(np.sum(x * hx)) < TOL
        assert abs(xaty - np.sum(x.astype(np.float64) * aty)) / np.abs(x * aty).sum() < 1e-6


# (n, expected Toeplitz FFT size): powers of two, and 3 x 2^k where smaller
TOEPLITZ_SIZES = [(100, 256), (256, 512), (513, 1536), (700, 1536), (768, 1536), (1024, 2048),
                  (1025, 3072), (1536, 3072), (2048, 4096), (2100, 6144), (2908, 6144)]


@pytest.mark.parametrize("n,M", TOEPLITZ_SIZES)
def test_toeplitz_large_with_given_psf(n, M):
    """Toeplitz FFT sizes up to 6144 on the register FFT (M = 1536 and 3072
    for images of 513 .. 768 and 1025 .. 1536 pixels; 6144 for 2100 and 2908,
    the padded grid of a 2048-pixel detector) against the FP64 oracle.

    A random even PSF is installed with set_psf (the operator only needs an
    even kernel), so sizes beyond the reach of the exact NUDFT are checked.
    """
    torch = _torch()
    from tomocam_b200.plan import Plan
    rng = np.random.default_rng(n)
    m1 = 2 * n - 1
    r = rng.standard_normal((m1, m1))
    psf = 0.5 * (r + r[::-1, ::-1])
    S = 3
    x = rng.standard_normal((S, n, n)).astype(np.float32)
    aty = rng.standard_normal((S, n, n)).astype(np.float32)
    with Plan(n, np.zeros(1, np.float32), psf=False) as pl:
        assert pl.info["toeplitz_m"] == M and pl.info["toeplitz_fast"] == 1
        pl.set_psf(psf)
        g, xhx, _ = pl.toeplitz_grad(torch.from_numpy(x).cuda(), torch.from_numpy(aty).cuda(),
                                     dots=True)
        hx = O.toeplitz_apply(x.astype(np.float64), psf)
        assert rel_l2(g.cpu().numpy(), hx - aty) < TOL
        assert abs(xhx - np.sum(x * hx)) <= TOL * np.abs(x * hx).sum()


@pytest.mark.parametrize("case", CASES[:2])
def test_nufft_grad_matches_toeplitz(plans, case):
    """gradient (NUFFT pair) == gradient2 (Toeplitz): test/gradient.cpp:76-83."""
    torch = _torch()
    pl, ang = plans[case]
    n, _ = case
    x = torch.from_numpy(phantom_stack(2, n, seed=4)).cuda()
    aty = torch.zeros_like(x)
    g1 = pl.nufft_grad(x, aty).cpu().numpy()
    g2 = pl.toeplitz_grad(x, aty).cpu().numpy()
    ref = O.gradient(x.cpu().numpy().astype(np.float64), np.zeros(x.shape), ang.astype(np.float64))
    assert rel_l2(g1, ref) < TOL
    assert rel_l2(g2, g1) < 2 * TOL


def test_lipschitz_matches_oracle(plans):
    pl, ang = plans[(32, 24)]
    psf = O.psf_kernel(32, ang.astype(np.float64))
    _, L = O.lipschitz_step(psf, 32)
    assert abs(pl.info["lipschitz"] - L) / L < 1e-5


@pytest.mark.parametrize("shape", [(1, 16, 16), (4, 17, 23), (5, 33, 40), (3, 8, 70)])
@pytest.mark.parametrize("sigma,p", [(10.0, 1.2), (0.5, 1.2), (0.05, 1.5)])
def test_qggmrf(shape, sigma, p):
    torch = _torch()
    from tomocam_b200.plan import qggmrf_grad
    rng = np.random.default_rng(0)
    x = rng.random(shape).astype(np.float32)
    g0 = rng.standard_normal(shape).astype(np.float32)
    g = qggmrf_grad(torch.from_numpy(x).cuda(), torch.from_numpy(g0).cuda(), sigma, p, 1.0)
    ref = g0.astype(np.float64) + O.qggmrf_grad(x.astype(np.float64), sigma, p)
    assert rel_l2(g.cpu().numpy(), ref) < TOL


def test_qggmrf_reference_golden():
    """Against outputs of the reference's own cpuTotalVar (test/tvd.cpp)."""
    torch = _torch()
    from tests.golden import load
    from tomocam_b200.plan import qggmrf_grad
    gold = load("qggmrf_ref")
    x = gold["x"]
    for k, (sigma, p) in enumerate(gold["params"]):
        g = torch.zeros(x.shape, dtype=torch.float32, device="cuda")
        qggmrf_grad(torch.from_numpy(x).cuda(), g, float(sigma), float(p), 1.0)
        assert rel_l2(g.cpu().numpy(), gold["out"][k]) < 2e-6


def test_empty_and_errors(plans):
    torch = _torch()
    from tomocam_b200 import _lib
    pl, _ = plans[(32, 24)]
    x = torch.zeros((0, 32, 32), device="cuda")
    assert pl.radon(x).shape == (0, 24, 32)
    with pytest.raises(ValueError):
        pl.radon(torch.zeros((1, 31, 31), device="cuda"))
    from tomocam_b200.plan import Plan
    with pytest.raises(_lib.TomocamError):
        Plan(2, np.zeros(4, np.float32))
    with pytest.raises(_lib.TomocamError):
        Plan(32, np.array([0.0, np.nan], np.float32))
    nopsf = Plan(32, np.zeros(4, np.float32), psf=False)
    with pytest.raises(_lib.TomocamError) as e:
        nopsf.toeplitz_grad(torch.zeros((1, 32, 32), device="cuda"))
    assert e.value.code == _lib.TC_ERR_STATE


@pytest.mark.parametrize("n,P", [(64, 90), (200, 150), (1024, 720)])
def test_autotuned_spreading_matches_default(n, P):
    """TC_PLAN_AUTOTUNE picks, by timing, the tile edge and sub-problem size
    of the tile path, the band-list chunk and NUFFT slices per chunk of the
    register-FFT path and the type-2 interpolation tiles; the
    back-projection and the NUFFT-pair gradient are unchanged up to the
    atomics' summation order, the projection (no atomics) exactly."""
    import torch
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(7)
    sino = torch.from_numpy(rng.standard_normal((2, P, n)).astype(np.float32)).cuda()
    x = torch.from_numpy(rng.standard_normal((2, n, n)).astype(np.float32)).cuda()
    with Plan(n, ang, psf=False) as a, Plan(n, ang, psf=False, autotune=True) as b:
        info = b.info
        assert info["spread_tile"] in (16, 32, 64)
        assert info["spread_max_points"] in (1024, 2048, 4096, 8192)
        assert a.info["spread_tile"] == 32 and a.info["spread_max_points"] == 2048
        assert a.info["band_chunk"] == 256
        assert info["band_chunk"] in (128, 256, 512, 1024)
        assert info["max_batch"] in (a.info["max_batch"], a.info["max_batch"] // 2)
        if a.info["interp_tile"]:
            assert a.info["interp_tile"] == 16 and a.info["interp_max_points"] == 256
            assert info["interp_tile"] in (16, 32)
            assert info["interp_max_points"] in (256, 1024, 4096)
        assert torch.equal(b.radon(x), a.radon(x))
        for ramp in (False, True):
            assert rel_l2(b.iradon(sino, ramp).cpu().numpy(), a.iradon(sino, ramp).cpu().numpy()) < 1e-6
        assert rel_l2(b.nufft_grad(x).cpu().numpy(), a.nufft_grad(x).cpu().numpy()) < 1e-6


@pytest.mark.parametrize("n,P", [(256, 180), (1000, 720)])
def test_band_spreading_register_form_is_exact(n, P):
    """NUFFT chunks of 8 complex lines (16 slices, two per line) spread with
    the register-accumulator band kernel, other chunk sizes with the
    shared-memory one; both add the same products to each cell in the same
    order, so back-projection and the NUFFT-pair gradient agree between
    max_batch 16 and 14 up to the order of the global atomic adds into bands
    split over several chunks (1e-6)."""
    torch = _torch()
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(11)
    sino = torch.from_numpy(rng.standard_normal((16, P, n)).astype(np.float32)).cuda()
    x = torch.from_numpy(rng.standard_normal((16, n, n)).astype(np.float32)).cuda()
    with Plan(n, ang, psf=False, max_batch=16) as a, Plan(n, ang, psf=False, max_batch=14) as b:
        assert a.info["band_chunk"] and b.info["band_chunk"]
        for ramp in (False, True):
            assert rel_l2(a.iradon(sino, ramp).cpu().numpy(), b.iradon(sino, ramp).cpu().numpy()) < 1e-6
        assert rel_l2(a.nufft_grad(x).cpu().numpy(), b.nufft_grad(x).cpu().numpy()) < 1e-6


@pytest.mark.parametrize("n", [600, 1100])
def test_power_of_two_toeplitz_flag(n):
    """TC_PLAN_POW2_TOEPLITZ keeps the power-of-two FFT size, with the same
    operator; the batched solver refuses a 3 x 2^k plan with a clear error."""
    torch = _torch()
    from tomocam_b200 import _lib
    from tomocam_b200.plan import BatchScan, Plan, mbir_batched
    rng = np.random.default_rng(n)
    m1 = 2 * n - 1
    r = rng.standard_normal((m1, m1))
    psf = 0.5 * (r + r[::-1, ::-1])
    x = torch.from_numpy(rng.standard_normal((2, n, n)).astype(np.float32)).cuda()
    ang = np.zeros(1, np.float32)
    with Plan(n, ang, psf=False) as p3, Plan(n, ang, psf=False, pow2_toeplitz=True) as p2:
        assert p3.info["toeplitz_m"] in (1536, 3072)
        assert p2.info["toeplitz_m"] in (2048, 4096)
        p3.set_psf(psf)
        p2.set_psf(psf)
        a, b = p3.toeplitz_grad(x).cpu().numpy(), p2.toeplitz_grad(x).cpu().numpy()
        assert rel_l2(a, b) < TOL
        with pytest.raises(_lib.TomocamError) as e:
            mbir_batched([BatchScan(p3, torch.zeros_like(x), 1.0, x.clone(), 5.0)], 1)
        assert e.value.code == _lib.TC_ERR_SHAPE and "POW2" in str(e.value)
