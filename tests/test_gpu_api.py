"""The reference-facing API (cTomocam / tomocam names) against the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import phantom_stack, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def test_radon_binding_2d_and_3d():
    from tomocam_b200 import cTomocam
    n, P = 40, 33
    ang = O.uniform_angles(P).astype(np.float32)
    img = phantom_stack(2, n, seed=1)
    out3 = cTomocam.radon(img, ang)
    out2 = cTomocam.radon(img[0], ang)
    ref = O.project(img.astype(np.float64), ang.astype(np.float64))
    assert out3.shape == (2, P, n) and out2.shape == (1, P, n)
    assert rel_l2(out3, ref) < TOL
    assert rel_l2(out2[0], ref[0]) < TOL


@pytest.mark.parametrize("center", [20.0, 17.4, 23.5])
def test_backproject_binding(center):
    from tomocam_b200 import cTomocam
    D, P = 40, 31
    ang = O.uniform_angles(P).astype(np.float32)
    sino = np.random.default_rng(2).standard_normal((2, P, D)).astype(np.float32)
    out = cTomocam.backproject(sino, ang, center)
    s2 = O.preproc(sino.astype(np.float64), center)
    ref = O.postproc(O.backproject(s2, ang.astype(np.float64)), D)
    assert out.shape == (2, D, D)
    assert rel_l2(out, ref) < TOL


def test_transform_module():
    import tomocam_b200 as tomocam
    n, P = 32, 20
    ang = O.uniform_angles(P).astype(np.float32)
    img = phantom_stack(1, n, seed=2)
    s = tomocam.radon(img, ang, 16.0, 1.5)
    assert rel_l2(s, O.project(img.astype(np.float64), ang.astype(np.float64))) < TOL
    b = tomocam.radon_adj(s, ang, 16.0)
    ref = O.postproc(O.backproject(O.preproc(s.astype(np.float64), 16.0), ang.astype(np.float64)), n)
    assert rel_l2(b, ref) < TOL


def test_calc_gradients_and_total_variation():
    from tomocam_b200 import modeling
    n, P = 32, 24
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    x = phantom_stack(2, n, seed=3)
    y = np.random.default_rng(4).standard_normal((2, P, n)).astype(np.float32)
    g = modeling.calc_gradients(x, y, ang)
    ref = O.backproject(O.project(x.astype(np.float64), a64) - y, a64)
    assert rel_l2(g, ref) < TOL
    g0 = np.random.default_rng(5).standard_normal(x.shape).astype(np.float32)
    g1 = modeling.update_total_variation(x, g0.copy(), smoothness=0.2)
    ref = g0 + O.qggmrf_grad(x.astype(np.float64), 5.0, 1.2)
    assert rel_l2(g1, ref) < TOL


def test_gradients_with_given_psf():
    from tests.golden import load
    from tomocam_b200.gradients import gradients
    gold = load("operators_n32")
    g = gradients(gold["x"], gold["aty"], gold["psf"])
    assert rel_l2(g, gold["toeplitz_grad"]) < TOL


def test_golden_operators():
    from tests.golden import load
    from tomocam_b200 import cTomocam
    from tomocam_b200.plan import Plan
    import torch
    gold = load("operators_n32")
    ang = gold["angles"]
    assert rel_l2(cTomocam.radon(gold["x"], ang), gold["radon"]) < TOL
    with Plan(32, ang) as pl:
        s = torch.from_numpy(gold["sino"]).cuda()
        assert rel_l2(pl.iradon(s).cpu().numpy(), gold["backproject"]) < TOL
        assert rel_l2(pl.iradon(s, ramp=True).cpu().numpy(), gold["fbp"]) < TOL
        assert rel_l2(pl.psf(), gold["psf"]) < 1e-10
        g = pl.toeplitz_grad(torch.from_numpy(gold["x"]).cuda(), torch.from_numpy(gold["aty"]).cuda())
        assert rel_l2(g.cpu().numpy(), gold["toeplitz_grad"]) < TOL


def test_set_num_of_gpus():
    from tomocam_b200 import cTomocam
    cTomocam.set_num_of_gpus(1)
    with pytest.raises(RuntimeError):
        cTomocam.set_num_of_gpus(0)


def test_device_memory_cache():
    """Buffers of a closed plan stay cached for the next plan of the same
    size (no new device memory is taken) until release_cached_memory()
    returns them; results are unchanged."""
    import torch
    from tomocam_b200.plan import Plan, release_cached_memory
    n, P = 512, 180
    ang = O.uniform_angles(P).astype(np.float32)
    x = torch.from_numpy(np.random.default_rng(3).standard_normal((4, n, n)).astype(np.float32)).cuda()
    release_cached_memory()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    with Plan(n, ang) as pl:
        y0 = pl.radon(x)
        g0 = pl.toeplitz_grad(x)
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 < free0  # the closed plan's blocks are held
    with Plan(n, ang) as pl:
        y1 = pl.radon(x)
        g1 = pl.toeplitz_grad(x)
        free2 = torch.cuda.mem_get_info()[0]
    assert free2 >= free1 - (64 << 20)  # served from the cache
    assert torch.equal(y0, y1) and torch.equal(g0, g1)
    release_cached_memory()
    assert torch.cuda.mem_get_info()[0] > free1

