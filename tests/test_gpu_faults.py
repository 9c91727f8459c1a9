"""Failure paths, injected on the host (no GPU fault is provoked).

The reference exits the process on these (src/gpu/utils.cuh:31-40 for CUDA
and allocation errors, src/mbir2.cpp:50-53 for a degenerate sinogram); the
library returns a status and the bindings raise:

* a device allocation that fails -> TC_ERR_ALLOC, injected through the
  library's TOMOCAM_B200_FAIL_ALLOC_ABOVE hook in a child process;
* a solve whose backtracking exhausts max_attempts -> TC_ERR_TIMEOUT, with
  the last accepted iterate written to the output;
* a sinogram holding NaN or Inf through cTomocam.mbir -> RuntimeError from
  TC_ERR_NAN, before any solve work.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import numpy as np, torch
from tomocam_b200 import _lib, cTomocam
from tomocam_b200.plan import Plan
torch.cuda.set_device(0)
ang = (np.arange(30) * np.pi / 30).astype(np.float32)
try:
    Plan(64, ang)
except _lib.TomocamError as e:
    assert e.code == _lib.TC_ERR_ALLOC, e.code
    assert "allocation" in str(e), str(e)
else:
    raise SystemExit("plan creation did not fail")
try:
    cTomocam.radon(np.ones((1, 64, 64), np.float32), ang)
except RuntimeError as e:
    assert "allocation" in str(e), str(e)
else:
    raise SystemExit("radon did not fail")
print("alloc-failure ok")
"""


def test_allocation_failure_is_reported():
    env = dict(os.environ, TOMOCAM_B200_FAIL_ALLOC_ABOVE="4096", PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "alloc-failure ok" in r.stdout


def test_exhausted_backtracking_reports_timeout_and_keeps_the_iterate():
    import torch
    from tests.test_gpu_mbir import _setup
    from tomocam_b200 import _lib
    from tomocam_b200.plan import Plan
    n = 32
    ang, a64, sino, aty, x0 = _setup(n, S=2, seed=3)
    sino, aty, x0 = sino * 1e-4, aty * 1e-4, x0 * 1e-4
    psf = O.psf_kernel(n, a64)
    step0, _ = O.lipschitz_step(psf, n)
    sino_sq = float(np.sum(sino ** 2))
    with Plan(n, ang) as pl:
        x = torch.from_numpy(x0.astype(np.float32)).cuda()
        start = x.clone()
        with pytest.raises(_lib.TomocamError) as e:
            pl.mbir_solve(torch.from_numpy(aty.astype(np.float32)).cuda(), sino_sq, x, 5, 1.0,
                          1.2, prior_weight=1e-3, step=2.5 * step0, max_attempts=3, inplace=True)
        # the oracle's run2 takes 3 attempts at iteration 0 and 4 at iteration 1
        assert e.value.code == _lib.TC_ERR_TIMEOUT
        assert "max_attempts" in str(e.value) and "iteration 1" in str(e.value)
        torch.cuda.synchronize()
        assert torch.isfinite(x).all()
        assert not torch.equal(x, start)   # the iterate reached so far was written


@pytest.mark.parametrize("bad", [float("nan"), float("inf"), -float("inf")])
def test_non_finite_sinogram_raises(bad):
    from tomocam_b200 import cTomocam
    D, P = 32, 20
    ang = O.uniform_angles(P).astype(np.float32)
    sino = np.abs(np.random.default_rng(1).standard_normal((2, P, D))).astype(np.float32)
    sino[1, 7, 11] = bad
    with pytest.raises(RuntimeError) as e:
        cTomocam.mbir(sino, ang, D / 2, 3, 5.0, 1e-4, 1e-4)
    assert "non-finite" in str(e.value)


def test_zero_sinogram_raises():
    from tomocam_b200 import cTomocam
    ang = O.uniform_angles(20).astype(np.float32)
    with pytest.raises(RuntimeError) as e:
        cTomocam.mbir(np.zeros((1, 20, 32), np.float32), ang, 16.0, 3, 5.0, 1e-4, 1e-4)
    assert "ZERO" in str(e.value)
