"""Batched MBIR over independent scans of uneven size (tc_mbir_batched):
each scan must reproduce its own single-volume solve and the FP64 oracle."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import phantom_stack, rel_l2

pytestmark = pytest.mark.gpu

# (n, angles, slices, sigma, prior weight): Toeplitz sizes 64, 128, 128, 256
SCANS = [(32, 40, 2, 5.0, 1.0), (48, 30, 1, 2.0, 0.5), (64, 50, 3, 5.0, 1.5), (96, 60, 1, 3.0, 1.0)]


def _scan_inputs(n, P, S, seed):
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    img = phantom_stack(S, n, seed=seed).astype(np.float64)
    sino = O.project(img, a64)
    sino = sino + 0.01 * sino.max() * np.random.default_rng(seed).standard_normal(sino.shape)
    aty = O.backproject(sino, a64).astype(np.float32)
    x0 = O.backproject(sino, a64, fbp=True).astype(np.float32)
    return ang, a64, sino, aty, x0


@pytest.fixture(scope="module")
def scans():
    import torch
    from tomocam_b200.plan import Plan
    out = []
    for i, (n, P, S, sigma, w) in enumerate(SCANS):
        ang, a64, sino, aty, x0 = _scan_inputs(n, P, S, seed=10 + i)
        out.append(dict(n=n, ang=ang, a64=a64, sino=sino, aty=aty, x0=x0, sigma=sigma, w=w,
                        sino_sq=float(np.sum(sino ** 2)), plan=Plan(n, ang),
                        aty_t=torch.from_numpy(aty).cuda()))
    yield out
    for s in out:
        s["plan"].close()


def _batch(scans, iters, use_graph=True, step_scale=0.0):
    import torch
    from tomocam_b200.plan import BatchScan, mbir_batched
    bs, xs = [], []
    for s in scans:
        x = torch.from_numpy(s["x0"]).cuda()
        step = step_scale / s["plan"].info["lipschitz"] if step_scale > 0 else 0.0
        bs.append(BatchScan(s["plan"], s["aty_t"], s["sino_sq"], x, s["sigma"], 1.2, s["w"], step))
        xs.append(x)
    hist = mbir_batched(bs, iters, use_graph=use_graph)
    return [x.cpu().numpy() for x in xs], hist


@pytest.mark.parametrize("use_graph", [True, False])
def test_batched_matches_single_solves(scans, use_graph):
    import torch
    iters = 6
    xb, hb = _batch(scans, iters, use_graph)
    for i, s in enumerate(scans):
        x, h = s["plan"].mbir_solve(s["aty_t"], s["sino_sq"], torch.from_numpy(s["x0"]).cuda(),
                                    iters, s["sigma"], 1.2, s["w"])
        assert rel_l2(xb[i], x.cpu().numpy()) < 1e-5
        np.testing.assert_array_equal(hb[i][:, 2], h[:, 2])
        np.testing.assert_allclose(hb[i][:, 0], h[:, 0], rtol=1e-5)


def test_batched_graph_equals_host_loop(scans):
    xg, hg = _batch(scans, 4, True)
    xp, hp = _batch(scans, 4, False)
    for a, b in zip(xg, xp):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(hg, hp)


def test_batched_matches_oracle_with_backtracking(scans):
    """Data scaled by 1e-4, prior weight 1e-3 and a step of 2.5 / L force
    rejected attempts (as in the single-volume backtracking test); every scan
    keeps its own backtracking sequence and matches the FP64 oracle's run2."""
    iters = 5
    small = []
    for s in scans:
        t = dict(s)
        t["aty"], t["aty_t"] = s["aty"] * 1e-4, s["aty_t"] * 1e-4
        t["x0"], t["sino_sq"], t["w"] = s["x0"] * 1e-4, s["sino_sq"] * 1e-8, 1e-3
        small.append(t)
    xb, hb = _batch(small, iters, step_scale=2.5)
    for i, s in enumerate(small):
        n = s["n"]
        psf = O.psf_kernel(n, s["a64"])
        aty = s["aty"].astype(np.float64)
        step = 2.5 / s["plan"].info["lipschitz"]

        def grad_fn(v):
            return O.gradient2(v, aty, psf) + O.qggmrf_grad(v, s["sigma"], 1.2, s["w"])

        def err_fn(v):
            return math.sqrt(O.function_value2(v, aty, psf, s["sino_sq"]))

        rec = O.Run2Record()
        ref = O.run2(s["x0"].astype(np.float64), iters, step, grad_fn, err_fn, rec)
        assert rel_l2(xb[i], ref) < 1e-4
        assert int(hb[i][:, 2].sum()) == rec.attempts
    assert hb[:, :, 2].sum() > len(scans) * iters  # backtracking happened
