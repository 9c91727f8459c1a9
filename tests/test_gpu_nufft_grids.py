"""Type-1 NUFFT (back-projection, ramp-filtered back-projection), type-2 NUFFT
(radon) and the NUFFT-pair gradient at every fine-grid size of the
register-FFT passes and one size beyond them (general engine), against the
oracle's FP64 ES NUFFT.

The fine grid is the smallest register-FFT length >= 2N: 256 (N = 100), 512,
1024, 1536, 2048, 3072, 4096 and 6144 (N = 2908, the padded grid of a
2048-pixel detector); N = 3200 takes the general 2,3,5,7-smooth engine.
The detector DFT runs directly on the register FFT when N is one of its
lengths (256, 1024, 1536, 2048) and as Bluestein's chirp convolution on the
next register length >= 2N - 1 otherwise (N = 2908 on 6144).
Operators are held to 1e-5 relative L2 error.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5
ES_TOL = 1e-10
SIZES = [(100, 40), (200, 40), (256, 40), (500, 30), (700, 30), (1000, 24), (1024, 24),
         (1400, 16), (1536, 16), (2000, 12), (2048, 8), (2908, 8), (3200, 6)]


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


@pytest.mark.parametrize("n,P", SIZES)
def test_backprojection_fine_grids(n, P):
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    sino = np.random.default_rng(n).standard_normal((2, P, n)).astype(np.float32)
    with Plan(n, ang, psf=False) as pl:
        nf = pl.info["nf"]
        assert nf >= 2 * n
        for ramp in (False, True):
            b = pl.iradon(_dev(sino), ramp=ramp).cpu().numpy()
            ref = O.backproject(sino.astype(np.float64), a64, fbp=ramp, method="es", tol=ES_TOL)
            assert rel_l2(b, ref) < TOL, (n, nf, ramp)


@pytest.mark.parametrize("n,P", SIZES)
def test_radon_fine_grids(n, P):
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(n + 3)
    x = rng.standard_normal((2, n, n)).astype(np.float32)
    with Plan(n, ang, psf=False) as pl:
        y = pl.radon(_dev(x)).cpu().numpy()
    ref = O.project(x.astype(np.float64), ang.astype(np.float64), "es", ES_TOL)
    assert rel_l2(y, ref) < TOL, (n, P)


@pytest.mark.parametrize("n,P", [(200, 40), (700, 30), (2908, 8)])
def test_nufft_gradient_fine_grids(n, P):
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(n + 1)
    x = rng.standard_normal((2, n, n)).astype(np.float32)
    aty = rng.standard_normal((2, n, n)).astype(np.float32)
    with Plan(n, ang, psf=False) as pl:
        g = pl.nufft_grad(_dev(x), _dev(aty)).cpu().numpy()
    ref = O.gradient(x.astype(np.float64), aty.astype(np.float64), ang.astype(np.float64),
                     method="es", tol=ES_TOL)
    assert rel_l2(g, ref) < TOL


@pytest.mark.parametrize("n,P", [(700, 30), (2908, 8)])
def test_adjoint_fine_grids(n, P):
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(n + 2)
    with Plan(n, ang, psf=False) as pl:
        x = _dev(rng.standard_normal((3, n, n)))
        y = _dev(rng.standard_normal((3, P, n)))
        ax = pl.radon(x).double()
        lhs = float((ax * y.double()).sum())
        rhs = float((x.double() * pl.iradon(y).double()).sum())
    assert abs(lhs - rhs) / (float(ax.norm()) * float(y.double().norm())) < 1e-5


@pytest.mark.parametrize("n,P,tol", [(200, 40, 1e-9), (700, 30, 1e-9), (4, 6, 0.0), (17, 9, 0.0)])
def test_wide_kernel_and_tiny_images(n, P, tol):
    """A tighter NUFFT tolerance (kernel width 10 > 8) takes the tile spreading
    on the column-major grid with the register-FFT passes; tiny images take
    the smallest fine grid (64) and a Bluestein detector DFT."""
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    rng = np.random.default_rng(n + 7)
    sino = rng.standard_normal((3, P, n)).astype(np.float32)
    x = rng.standard_normal((3, n, n)).astype(np.float32)
    with Plan(n, ang, nufft_tol=tol, psf=False) as pl:
        if tol:
            assert pl.info["kernel_width"] > 8
        b = pl.iradon(_dev(sino)).cpu().numpy()
        y = pl.radon(_dev(x)).cpu().numpy()
    assert rel_l2(b, O.backproject(sino.astype(np.float64), a64, method="es", tol=ES_TOL)) < TOL
    assert rel_l2(y, O.project(x.astype(np.float64), a64, "es", ES_TOL)) < TOL


@pytest.mark.parametrize("tol,w", [(1e-3, 4), (1e-5, 6), (1e-7, 8)])
def test_kernel_widths_on_tiles_and_register_bands(tol, w):
    """Other NUFFT tolerances change the kernel width W, a template parameter
    of the tiled interpolation and of the register band spreading: radon and
    back-projection of 16 slices (one chunk of 8 paired lines:
    k_t2_interp_tile<16, W>, k_spread_band8<W>) against the accurate oracle
    within the requested tolerance, and the back-projection against chunks
    of 14 slices (7 lines: the shared-memory band kernel) to 1e-6."""
    from tomocam_b200.plan import Plan
    n, P = 300, 120
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    rng = np.random.default_rng(w)
    sino = rng.standard_normal((16, P, n)).astype(np.float32)
    x = rng.standard_normal((16, n, n)).astype(np.float32)
    with Plan(n, ang, nufft_tol=tol, psf=False) as pl, \
            Plan(n, ang, nufft_tol=tol, psf=False, max_batch=14) as p7:
        assert pl.info["kernel_width"] == w and pl.info["max_batch"] == 16
        assert pl.info["paired_nufft"] == 1
        assert pl.info["interp_tile"] and pl.info["band_chunk"]
        b = pl.iradon(_dev(sino)).cpu().numpy()
        b7 = p7.iradon(_dev(sino)).cpu().numpy()
        y = pl.radon(_dev(x)).cpu().numpy()
    bound = max(20 * tol, TOL)
    assert rel_l2(b, O.backproject(sino.astype(np.float64), a64, method="es", tol=ES_TOL)) < bound
    assert rel_l2(y, O.project(x.astype(np.float64), a64, "es", ES_TOL)) < bound
    assert rel_l2(b, b7) < 1e-6


@pytest.mark.parametrize("S", [5, 6, 7, 13, 21])
def test_chunk_remainders(S):
    """NUFFT chunks hold up to 16 slices as 8 complex lines of two slices;
    5, 7, 13 and 21 (= 16 + 5) slices end on a line with one slice (the
    imaginary part zero), 6 on full lines, and the band-spreading kernels
    run for 3 to 8 lines per chunk."""
    from tomocam_b200.plan import Plan
    n, P = 64, 45
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    rng = np.random.default_rng(S)
    sino = rng.standard_normal((S, P, n)).astype(np.float32)
    x = rng.standard_normal((S, n, n)).astype(np.float32)
    with Plan(n, ang, psf=False) as pl:
        assert pl.info["max_batch"] == 16 and pl.info["paired_nufft"] == 1
        b = pl.iradon(_dev(sino)).cpu().numpy()
        y = pl.radon(_dev(x)).cpu().numpy()
        g = pl.nufft_grad(_dev(x)).cpu().numpy()
    assert rel_l2(b, O.backproject(sino.astype(np.float64), a64)) < TOL
    assert rel_l2(y, O.project(x.astype(np.float64), a64)) < TOL
    x64 = x.astype(np.float64)
    ref = O.gradient(x64, np.zeros_like(x64), a64, method="es", tol=ES_TOL)
    assert rel_l2(g, ref) < TOL


@pytest.mark.parametrize("n,P,S", [(256, 180, 5), (301, 90, 4), (1000, 360, 3), (2048, 64, 2)])
def test_paired_lines_match_unpaired(n, P, S):
    """Two slices per complex line (the default on the register-FFT path)
    against one slice per line (TC_PLAN_UNPAIRED): radon, back-projection
    with and without the ramp, and the NUFFT-pair gradient agree to 1e-6,
    for even detector counts (the j = 0 sample and its mirror point) and an
    odd one (301: no mirror points)."""
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(n + S)
    sino = _dev(rng.standard_normal((S, P, n)))
    x = _dev(rng.standard_normal((S, n, n)))
    with Plan(n, ang, psf=False) as a, Plan(n, ang, psf=False, paired=False) as b:
        assert a.info["paired_nufft"] == 1 and b.info["paired_nufft"] == 0
        assert a.info["max_batch"] == 2 * b.info["max_batch"]
        assert rel_l2(a.radon(x).cpu().numpy(), b.radon(x).cpu().numpy()) < 1e-6
        for ramp in (False, True):
            assert rel_l2(a.iradon(sino, ramp).cpu().numpy(),
                          b.iradon(sino, ramp).cpu().numpy()) < 1e-6
        assert rel_l2(a.nufft_grad(x).cpu().numpy(), b.nufft_grad(x).cpu().numpy()) < 1e-6


def test_paired_slices_do_not_mix():
    """The two slices of a line separate exactly up to rounding: next to a
    non-zero slice, a zero slice projects, back-projects and takes the
    NUFFT gradient to values below 1e-6 of its neighbour's."""
    from tomocam_b200.plan import Plan
    n, P = 512, 240
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(3)
    x = np.zeros((2, n, n), np.float32)
    x[0] = rng.standard_normal((n, n))
    sino = np.zeros((2, P, n), np.float32)
    sino[1] = rng.standard_normal((P, n))
    with Plan(n, ang, psf=False) as pl:
        assert pl.info["paired_nufft"] == 1
        y = pl.radon(_dev(x)).cpu().numpy()
        g = pl.nufft_grad(_dev(x)).cpu().numpy()
        b = pl.iradon(_dev(sino), True).cpu().numpy()
    assert np.abs(y[1]).max() < 1e-6 * np.abs(y[0]).max()
    assert np.abs(g[1]).max() < 1e-6 * np.abs(g[0]).max()
    assert np.abs(b[0]).max() < 1e-6 * np.abs(b[1]).max()
