"""The FP64 oracle, pinned before it is trusted (CPU only).

* the prior against the reference's own CPU implementation (cpuTotalVar,
  test/tvd.cpp:40-75) through the committed golden fixture;
* the NUFFT restatement against the exact non-uniform DFT;
* the reference's identity tests: gradient == Toeplitz gradient
  (test/gradient.cpp:76-83, test/toeplitz.cpp:84-85) and the objective forms
  (test/error.cpp:77-82);
* run2's control flow (src/optimize.h:96-154).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import load
from tests.helpers import rel_l2


def test_qggmrf_matches_reference_cpu_code():
    g = load("qggmrf_ref")
    x = g["x"].astype(np.float64)
    for k, (sigma, p) in enumerate(g["params"]):
        ref = g["out"][k].astype(np.float64)
        assert rel_l2(O.qggmrf_grad(x, float(sigma), float(p)), ref) < 1e-6
        assert rel_l2(O.qggmrf_grad(x, float(sigma), float(p), use_core=False), ref) < 1e-6


def test_reference_shim_if_built():
    """When the reference was compiled here (oracle/_ref), recheck it live."""
    import ctypes
    import os
    path = os.path.join(os.path.dirname(O.__file__), "_ref", "libref_tvd.so")
    if not os.path.exists(path):
        pytest.skip("reference shim not built (make -C oracle ref)")
    lib = ctypes.CDLL(path)
    fp = ctypes.POINTER(ctypes.c_float)
    lib.ref_cpu_total_var.argtypes = [fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_float]
    x = np.random.default_rng(0).random((3, 9, 14)).astype(np.float32)
    out = np.empty_like(x)
    assert lib.ref_cpu_total_var(x.ctypes.data_as(fp), out.ctypes.data_as(fp), 3, 9, 14, 2.0, 1.3) == 0
    assert rel_l2(O.qggmrf_grad(x.astype(np.float64), 2.0, 1.3), out) < 1e-6


@pytest.mark.parametrize("n,P", [(16, 12), (17, 9), (24, 20)])
def test_es_nufft_matches_exact(n, P):
    rng = np.random.default_rng(n)
    x, y = O.polar_grid(P, n, O.uniform_angles(P))
    f = rng.standard_normal((2, n, n)) + 1j * rng.standard_normal((2, n, n))
    c = rng.standard_normal((2, P * n)) + 1j * rng.standard_normal((2, P * n))
    assert rel_l2(O.es_type2(f, x, y, 1e-12), O.nudft_type2(f, x, y)) < 1e-10
    assert rel_l2(O.es_type1(c, x, y, n, 1e-12), O.nudft_type1(c, x, y, n)) < 1e-10
    # the tolerance the GPU operators run at
    assert rel_l2(O.es_type1(c, x, y, n, 1e-6), O.nudft_type1(c, x, y, n)) < 5e-6


@pytest.mark.parametrize("n,P", [(16, 12), (21, 15)])
def test_project_backproject_adjoint(n, P):
    rng = np.random.default_rng(1)
    ang = O.uniform_angles(P)
    x = rng.standard_normal((2, n, n))
    y = rng.standard_normal((2, P, n))
    lhs = np.sum(O.project(x, ang) * y)
    rhs = np.sum(x * O.backproject(y, ang))
    assert abs(lhs - rhs) < 1e-10 * np.linalg.norm(x) * np.linalg.norm(y) * n


@pytest.mark.parametrize("n,P", [(16, 12), (21, 15), (32, 24)])
def test_gradient_equals_toeplitz_gradient(n, P):
    ang = O.uniform_angles(P)
    x = np.random.default_rng(2).standard_normal((2, n, n))
    aty = np.random.default_rng(3).standard_normal((2, n, n))
    psf = O.psf_kernel(n, ang)
    assert rel_l2(O.gradient2(x, aty, psf), O.gradient(x, aty, ang)) < 1e-12


def test_objective_forms_agree_for_odd_n():
    """|Ax-y|^2 == x.Hx - 2x.A^Ty + |y|^2 (test/error.cpp:77-82) when N is odd.

    For even N the reference's H = Re(NUFFT1 NUFFT2)/N^3 differs from A^T A
    (A takes the real part after the detector IFFT, and the even-N mode set
    [-N/2, N/2) is not symmetric), so the forms differ; the solver uses the H
    form throughout, as the reference does.
    """
    n, P = 21, 17
    ang = O.uniform_angles(P)
    x = O.ellipse_phantom(n, 5, 1)[None]
    y = O.project(x, ang) + 0.01
    psf = O.psf_kernel(n, ang)
    aty = O.backproject(y, ang)
    f1 = O.function_value(x, y, ang)
    f2 = O.function_value2(x, aty, psf, float(np.sum(y * y)))
    assert abs(f1 - f2) / f1 < 1e-9


def test_psf_is_even():
    n, P = 18, 14
    psf = O.psf_kernel(n, O.uniform_angles(P))
    assert np.allclose(psf, psf[::-1, ::-1], rtol=0, atol=1e-9 * np.abs(psf).max())


def test_preproc_postproc_roundtrip():
    D = 40
    sino = np.random.default_rng(0).random((2, 5, D))
    for center in (20.0, 13.6, 27.5, 19.5):
        npad, off = O.preproc_params(D, center)
        s2 = O.preproc(sino, center)
        assert s2.shape == (2, 5, D + 2 * npad)
        # undo the roll and the padding
        back = np.roll(s2, off, axis=-1)[:, :, npad:npad + D]
        assert np.array_equal(back, sino)
    x = np.random.default_rng(1).random((1, D + 2 * npad, D + 2 * npad))
    assert O.postproc(x, D).shape == (1, D, D)
    assert np.array_equal(O.postproc(O.pad2d_symmetric(x[:, :D, :D], 2 * npad), D), x[:, :D, :D])


def test_preproc_params_follow_reference_rounding():
    # std::round rounds halves away from zero; npad = int(0.42 n) / 2
    assert O.preproc_params(2048, 1024.0) == (430, 0)
    assert O.preproc_params(2048, 1023.5) == (430, 0)
    assert O.preproc_params(256, 128.0) == (53, 0)
    assert O.preproc_params(100, 10.0) == (40, 40)


def test_run2_quirks():
    """After an accepted step x == sol, so the next y carries no momentum."""
    calls = []

    def grad_fn(y):
        calls.append(y.copy())
        return 2.0 * (y - 3.0)

    def err_fn(v):
        return math.sqrt(float(np.sum((v - 3.0) ** 2)))

    rec = O.Run2Record()
    O.run2(np.zeros(4), 3, 0.1, grad_fn, err_fn, rec)
    # every attempt accepted: y of attempt k equals the solution of attempt k-1
    assert rec.attempts == 3
    assert np.allclose(calls[1], 0.6) and np.allclose(calls[2], 0.6 + 0.2 * 2.4)


def test_golden_operators_match_live_oracle():
    g = load("operators_n32")
    a64 = g["angles"].astype(np.float64)
    assert rel_l2(O.project(g["x"].astype(np.float64), a64), g["radon"]) < 1e-12
    assert rel_l2(O.psf_kernel(32, a64), g["psf"]) < 1e-12


def test_toeplitz_cache_is_the_same_arithmetic():
    ang = O.uniform_angles(14)
    psf = O.psf_kernel(12, ang)
    rng = np.random.default_rng(3)
    x, aty = rng.random((2, 12, 12)), rng.random((2, 12, 12))
    c = O.ToeplitzCache(psf)
    for _ in range(2):   # second pass served from the cache
        assert np.array_equal(c.gradient2(x, aty), O.gradient2(x, aty, psf))
        assert c.function_value2(x, aty, 3.5) == O.function_value2(x, aty, psf, 3.5)
