"""oracle.run2 pinned to the reference's own Optimizer::run2 (CPU only).

The reference's solver (src/optimize.h:96-154) is compiled from the reference
tree into oracle/_ref/libref_run2.so and driven with the FP64 oracle's
gradient (gradient2 + qGGMRF) and objective (sqrt function_value2), as
src/mbir2.cpp:114-137 wires them.  Its results, gradient-evaluation counts
and the full sequence of objective values it requested are committed in
tests/golden/run2_ref.npz; the oracle's restatement must reproduce all three
on a plain case and on a case that backtracks.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import load
from tests.golden.make_golden import run2_callbacks
from tests.helpers import rel_l2
from tests.refbuild import ref_run2, run2_lib

CASES = ("plain", "backtrack")


def _case(name):
    g = load("run2_ref")
    keys = ("x0", "aty", "psf", "sino_sq", "sigma", "p", "weight", "step", "iters")
    c = {k: g[f"{name}_{k}"] for k in keys}
    for k in ("sino_sq", "sigma", "p", "weight", "step"):
        c[k] = float(c[k])
    c["iters"] = int(c["iters"])
    return c, g[f"{name}_out"], int(g[f"{name}_attempts"]), g[f"{name}_errs"]


def _oracle(c):
    grad_fn, err_fn = run2_callbacks(c)
    errs = []

    def err_logged(v):
        e = err_fn(v)
        errs.append(e)
        return e

    rec = O.Run2Record()
    x = O.run2(c["x0"], c["iters"], c["step"], grad_fn, err_logged, rec)
    return x, rec, np.array(errs)


@pytest.mark.parametrize("name", CASES)
def test_oracle_run2_reproduces_reference_run2(name):
    c, ref_out, ref_attempts, ref_errs = _case(name)
    x, rec, errs = _oracle(c)
    assert rec.attempts == ref_attempts
    assert errs.shape == ref_errs.shape
    assert np.allclose(errs, ref_errs, rtol=1e-12, atol=0.0)
    assert rel_l2(x, ref_out) < 1e-12


def test_backtracking_case_backtracks():
    c, _, attempts, _ = _case("backtrack")
    assert attempts > c["iters"]          # rejected attempts happened
    c, _, attempts, _ = _case("plain")
    assert attempts == c["iters"]         # every first attempt accepted


@pytest.mark.parametrize("name", CASES)
def test_reference_run2_live_if_built(name):
    """When oracle/_ref was compiled here, rerun the reference and recheck the fixture."""
    if run2_lib() is None:
        pytest.skip("reference solver not built (make -C oracle ref)")
    c, ref_out, ref_attempts, ref_errs = _case(name)
    grad_fn, err_fn = run2_callbacks(c)
    x, attempts, errs = ref_run2(c["x0"], c["iters"], c["step"], grad_fn, err_fn)
    assert attempts == ref_attempts
    assert np.allclose(errs, ref_errs, rtol=1e-12, atol=0.0)
    assert rel_l2(x, ref_out) < 1e-12
