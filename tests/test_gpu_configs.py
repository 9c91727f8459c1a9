"""The benchmark workloads' own depth and sizes against the FP64 oracle.

* Full-volume MBIR: slices 126-129 of the seeded 256 x 2048^2 foam (2000
  spheres), 1969 angles, Poisson noise at 1e4 counts, qGGMRF p = 1.2,
  sigma = 100 (the reference's default smoothness 0.01), all 50
  iterations; the image and every iteration's objective are held to 1e-4.
* Uneven batch: six independent scans drawn from the uneven-batch workload's
  sizes (n = 1024 with 1500 angles and n = 384 with 360 among them), seeded
  ellipse phantoms with 1 % noise, each with its own PSF, step and prior
  weight beta ~ U[0.1, 2], solved together by tc_mbir_batched for 50
  iterations; each scan's image is held to 1e-4.  The workload's prior
  "sigma = 0.05" is read as the API's smoothness (sigma = 1/0.05 = 20), as
  for the one-slice workload: with sigma = 0.05 itself the step 1/L ignores
  the prior's curvature and the iteration is unstable in any precision.

The sinograms, A^T y and the FBP start come from the product's operators
(held to 1e-5 against the oracle elsewhere); from there the product's solver
and the oracle's run2 (FP64 PSF, FP64 Toeplitz products and prior) start
from the same FP32 inputs.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

TOL_RECON = 1e-4
ES_TOL = 1e-10


def _oracle_solve(x0, aty, sino_sq, psf, iters, step, sigma, weight=1.0):
    cache = O.ToeplitzCache(psf)

    def grad_fn(v):
        return cache.gradient2(v, aty) + O.qggmrf_grad(v, sigma, 1.2, weight)

    def err_fn(v):
        return math.sqrt(cache.function_value2(v, aty, sino_sq))

    rec = O.Run2Record()
    x = O.run2(x0, iters, step, grad_fn, err_fn, rec)
    return x, rec


def test_full_volume_foam_all_50_iterations():
    import torch
    from tomocam_b200 import phantom
    from tomocam_b200.plan import Plan
    S, n, P, sigma, iters = 4, 2048, 1969, 100.0, 50
    ang = O.uniform_angles(P).astype(np.float32)
    vol = phantom.foam_volume(S, n, 2000, seed=0, total=256, first=126)
    with Plan(n, ang) as pl:
        y = phantom.transmission_noise(pl.radon(vol), 1e4, 3.0, seed=0)
        y /= y.max()
        aty = pl.iradon(y)
        x0 = pl.iradon(y, ramp=True)
        sino_sq = float((y.double() ** 2).sum())
        step = min(1.0 / pl.info["lipschitz"], 1.0)
        x, hist = pl.mbir_solve(aty, sino_sq, x0, iters, sigma, 1.2, step=step)
        torch.cuda.synchronize()
        aty64 = aty.cpu().numpy().astype(np.float64)
        x064 = x0.cpu().numpy().astype(np.float64)
        x = x.cpu().numpy()
    psf = O.psf_kernel(n, ang.astype(np.float64), "es", ES_TOL)
    step_ref, _ = O.lipschitz_step(psf, n)
    assert abs(step_ref - step) <= 1e-6 * step
    ref, rec = _oracle_solve(x064, aty64, sino_sq, psf, iters, step, sigma)
    err = rel_l2(x, ref)
    print(f"foam 4 x 2048^2, 50 iterations: rel.err {err:.2e}, attempts {rec.attempts}")
    assert err < TOL_RECON
    assert int(hist[:, 2].sum()) == rec.attempts
    err_ref = np.array([e for _, e, _ in rec.iters])
    assert rel_l2(hist[:, 0], err_ref) < TOL_RECON


# (n, angles): drawn from the uneven-batch sizes, the largest and a small one first
BATCH4 = [(1024, 1500), (384, 360), (256, 180), (512, 720), (768, 1024), (256, 1500)]


def test_uneven_batch_50_iterations_per_scan_error():
    import torch
    from tomocam_b200 import phantom
    from tomocam_b200.plan import BatchScan, Plan, mbir_batched
    iters, sigma = 50, 20.0
    betas = np.random.default_rng(4).uniform(0.1, 2.0, len(BATCH4))
    plans, scans, inputs = [], [], []
    try:
        for i, (n, P) in enumerate(BATCH4):
            ang = O.uniform_angles(P).astype(np.float32)
            pl = Plan(n, ang, pow2_toeplitz=True)   # the batched passes take powers of two
            plans.append(pl)
            img = phantom.ellipse_slices(1, n, 10, seed=40 + i)
            y = pl.radon(img)
            g = torch.Generator(device="cuda").manual_seed(40 + i)
            y = y + 0.01 * y.max() * torch.randn(y.shape, device="cuda", generator=g)
            y /= y.max()
            aty = pl.iradon(y)
            x = pl.iradon(y, ramp=True)
            sino_sq = float((y.double() ** 2).sum())
            step = min(1.0 / pl.info["lipschitz"], 1.0)
            inputs.append((ang, aty.cpu().numpy().astype(np.float64),
                           x.cpu().numpy().astype(np.float64), sino_sq, step))
            scans.append(BatchScan(pl, aty, sino_sq, x, sigma, 1.2, float(betas[i]), step))
        hist = mbir_batched(scans, iters, use_graph=True)
        torch.cuda.synchronize()
        outs = [s.x.cpu().numpy() for s in scans]
    finally:
        for pl in plans:
            pl.close()
    errs = []
    for i, (n, P) in enumerate(BATCH4):
        ang, aty, x0, sino_sq, step = inputs[i]
        psf = O.psf_kernel(n, ang.astype(np.float64), "es", ES_TOL)
        ref, rec = _oracle_solve(x0, aty, sino_sq, psf, iters, step, sigma, float(betas[i]))
        errs.append(rel_l2(outs[i], ref))
        assert int(hist[i][:, 2].sum()) == rec.attempts, (n, P)
    print("per-scan rel.err vs FP64:", ", ".join(f"{n}/{P}: {e:.2e}"
                                                 for (n, P), e in zip(BATCH4, errs)))
    assert max(errs) < TOL_RECON
