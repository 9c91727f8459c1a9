"""tc_toeplitz_grad_noalloc: the Toeplitz gradient for callers that cannot
allocate device memory -- applications whose own pool allocator owns the
GPU's memory and forbid a library to call cudaMalloc, which could fail
against the full pool or synchronise the device mid-pipeline.

It must give the same gradient and dot products as the allocating entry
point tc_toeplitz_grad, on two calls in a row (the calls share one scratch
array, which keeps the previous call's contents), agree with the FP64
oracle, accept every image up to 1024 x 1024, and refuse plans whose
slice-pair workspace does not fit the fixed 32 MiB scratch.  This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _noalloc(pl, x, aty, g, S):
    import torch
    from tomocam_b200 import _lib
    a, b = ctypes.c_double(0.0), ctypes.c_double(0.0)
    _lib.call("tc_toeplitz_grad_noalloc", pl._h, ctypes.c_void_p(x.data_ptr()),
              ctypes.c_void_p(aty.data_ptr()) if aty is not None else None,
              ctypes.c_void_p(g.data_ptr()), S, ctypes.byref(a), ctypes.byref(b),
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return a.value, b.value


SCRATCH = 32 << 20


def _fits(n, M):
    """The entry point's own rule: one slice pair's workspace, partial sums
    and alignment within the scratch minus its 256-byte header."""
    return n * M * 8 + 16 * n + 256 <= SCRATCH - 256


@pytest.mark.parametrize("n,P,S", [(64, 45, 5), (200, 120, 2), (333, 90, 3), (1024, 32, 2)])
def test_noalloc_matches_allocating_entry_point(n, P, S):
    import torch
    from oracle import oracle as O
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(n)
    x = torch.from_numpy(rng.standard_normal((S, n, n)).astype(np.float32)).cuda()
    aty = torch.from_numpy(rng.standard_normal((S, n, n)).astype(np.float32)).cuda()
    with Plan(n, ang) as pl:
        ref, rhx, raty = pl.toeplitz_grad(x, aty, dots=True)
        ref = ref.cpu().numpy()
        for _ in range(2):  # the second call reuses the scratch left by the first
            g = torch.full_like(x, float("nan"))
            xhx, xaty = _noalloc(pl, x, aty, g, S)
            assert rel_l2(g.cpu().numpy(), ref) < TOL
            assert abs(xhx - rhx) <= TOL * abs(rhx)
            assert abs(xaty - raty) <= TOL * abs(raty)
        g = torch.empty_like(x)
        _noalloc(pl, x, None, g, S)
        ref0 = pl.toeplitz_grad(x).cpu().numpy()
        assert rel_l2(g.cpu().numpy(), ref0) < TOL


def test_noalloc_matches_fp64_oracle():
    import torch
    from oracle import oracle as O
    from tomocam_b200.plan import Plan
    n, P, S = 48, 40, 3
    ang = O.uniform_angles(P).astype(np.float32)
    rng = np.random.default_rng(7)
    x = rng.standard_normal((S, n, n)).astype(np.float32)
    aty = rng.standard_normal((S, n, n)).astype(np.float32)
    psf = O.psf_kernel(n, ang.astype(np.float64))
    want = O.gradient2(x.astype(np.float64), aty.astype(np.float64), psf)
    dx, da = torch.from_numpy(x).cuda(), torch.from_numpy(aty).cuda()
    with Plan(n, ang) as pl:
        for _ in range(2):
            g = torch.full_like(dx, float("nan"))
            xhx, xaty = _noalloc(pl, dx, da, g, S)
            assert rel_l2(g.cpu().numpy(), want) < TOL
            hx = want + aty.astype(np.float64)
            assert abs(xhx - float(np.sum(x * hx))) <= TOL * abs(float(np.sum(x * hx)))


@pytest.mark.parametrize("n", [1025, 1400, 1600])
def test_noalloc_rejects_images_beyond_the_scratch(n):
    """Beyond 1024 pixels the plan's FFT size decides: a plan whose pair does
    not fit fails with TC_ERR_SHAPE before any launch (sizes that fit are
    exercised by the tests above)."""
    import torch
    from tomocam_b200 import _lib
    from tomocam_b200.plan import Plan
    with Plan(n, np.zeros(2, np.float32), psf=False) as pl:
        M = pl.info["toeplitz_m"]
        x = torch.zeros((1, n, n), device="cuda")
        if _fits(n, M):
            pytest.skip(f"n = {n} fits the scratch with M = {M}")
        with pytest.raises(_lib.TomocamError) as e:
            _noalloc(pl, x, None, torch.empty_like(x), 1)
        assert e.value.code == _lib.TC_ERR_SHAPE
        assert "scratch" in str(e.value)


def test_noalloc_limit_rule():
    """Every N <= 1024 fits: the largest FFT size there is 2048."""
    assert _fits(1024, 2048)
    assert not _fits(1025, 4096)
