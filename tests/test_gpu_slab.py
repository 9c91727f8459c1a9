"""Slab sharding on one GPU: a volume split into consecutive slabs, solved in
lockstep with halo exchange and summed step tests (tomocam_b200.slab),
against the whole-volume solve of the same inputs.  The sharded solve runs
the same kernels; only the FP32/FP64 summation order of the step-test sums
differs, so the attempts are the same and the results agree to FP32
rounding."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import phantom_stack, rel_l2

pytestmark = pytest.mark.gpu


def _data(n, P, S, seed, scale=1.0):
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    img = phantom_stack(S, n, seed=seed).astype(np.float64)
    sino = O.project(img, a64)
    sino = sino + 0.01 * sino.max() * np.random.default_rng(seed).standard_normal(sino.shape)
    sino = sino * scale
    aty = O.backproject(sino, a64)
    x0 = O.backproject(sino, a64, fbp=True)
    return ang, float(np.sum(sino ** 2)), aty.astype(np.float32), x0.astype(np.float32)


def _compare(split, n=40, P=30, seed=3, iters=6, sigma=3.0, weight=1.0, step=0.0, scale=1.0):
    import torch
    from tomocam_b200.plan import Plan
    from tomocam_b200.slab import Slab, solve_slabs_local
    S = sum(split)
    ang, sino_sq, aty, x0 = _data(n, P, S, seed, scale)
    aty_d = torch.from_numpy(np.ascontiguousarray(aty)).cuda()
    x0_d = torch.from_numpy(np.ascontiguousarray(x0)).cuda()
    with Plan(n, ang) as pl:
        xw, hw = pl.mbir_solve(aty_d, sino_sq, x0_d.clone(), iters, sigma, 1.2, prior_weight=weight,
                               step=step, use_graph=False)
        bounds = np.cumsum((0,) + tuple(split))
        slabs = [Slab(pl, aty_d[a:b].contiguous(), sino_sq, x0_d[a:b].contiguous(), iters, sigma, 1.2,
                      prior_weight=weight, step=step) for a, b in zip(bounds[:-1], bounds[1:])]
        res = solve_slabs_local(slabs)
        for s in slabs:
            s.close()
    xs = torch.cat([x for x, _ in res]).cpu().numpy()
    for _, h in res:
        assert np.array_equal(h[:, 2], hw[:, 2])          # same attempts per iteration
        assert rel_l2(h[:, 0], hw[:, 0]) < 1e-6            # objective
    assert rel_l2(xs, xw.cpu().numpy()) < 1e-5
    return hw


@pytest.mark.parametrize("split", [(7,), (3, 4), (2, 2, 3), (1, 5, 1)])
def test_slabs_match_whole_volume(split):
    _compare(split)


def test_slabs_match_whole_volume_with_backtracking():
    """Rejected attempts (x and sol then differ, so both buffers' halos are
    exchanged): data scaled by 1e-4 and a step of 2.5/L as in the solver's
    backtracking test."""
    import torch  # noqa: F401
    from tomocam_b200.plan import Plan
    n, P = 40, 30
    ang, _, _, _ = _data(n, P, 1, 0)
    psf = O.psf_kernel(n, ang.astype(np.float64))
    step0, _ = O.lipschitz_step(psf, n)
    hw = _compare((3, 2, 3), n=n, P=P, seed=5, iters=5, sigma=1.0, weight=1e-3, step=2.5 * step0,
                  scale=1e-4)
    assert hw[:, 2].sum() > len(hw)                        # the whole-volume solve did backtrack
