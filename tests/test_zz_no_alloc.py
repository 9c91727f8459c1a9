"""tc_toeplitz_grad_noalloc: the Toeplitz gradient for callers that cannot
allocate device memory (for example code running inside a CUDA graph
capture, or an application whose own pool allocator owns the GPU's memory).

It must give the same gradient and dot products as the allocating entry
point tc_toeplitz_grad, on repeated calls (the calls share one scratch
array), and refuse plans whose slice-pair workspace does not fit the fixed
32 MiB scratch.  This file is collected last so that a run stopping at the
first failure has already run every other test.
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


@pytest.mark.parametrize("n,P,S", [(64, 45, 5), (200, 120, 2), (333, 90, 3)])
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


def test_noalloc_rejects_images_beyond_the_scratch():
    import torch
    from tomocam_b200 import _lib
    from tomocam_b200.plan import Plan
    n = 1600
    with Plan(n, np.zeros(2, np.float32), psf=False) as pl:
        x = torch.zeros((1, n, n), device="cuda")
        with pytest.raises(_lib.TomocamError) as e:
            _noalloc(pl, x, None, torch.empty_like(x), 1)
        assert e.value.code == _lib.TC_ERR_SHAPE
        assert "scratch" in str(e.value)
