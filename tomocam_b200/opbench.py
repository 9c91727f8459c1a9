"""Operator benchmark: time radon, back-projection, the Toeplitz gradient, the
qGGMRF update and the MBIR solve on synthetic data, one JSON line.

    python -m tomocam_b200.opbench                      # operator-pair workload
    python -m tomocam_b200.opbench --op toeplitz --n 2048 --slices 2 --psf random
    python -m tomocam_b200.opbench --op solve --n 2048 --slices 256 --iters 3 --psf random
    python -m tomocam_b200.opbench --op autograd --n 768 --inner 512 --nproj 720 --slices 32
    python -m tomocam_b200.opbench --op batched --scans 48 --iters 50

Default workload (the operator-pair throughput configuration): 64 slices of
1024 x 1024 ellipse phantoms with N(0, 0.01) texture embedded in 1536 x 1536
(the operators need the image width to equal the detector count), 1500
angles on [0, pi), 1536 detector pixels; radon, back-projection and the
Toeplitz gradient are each timed with CUDA events (after warm-up, inputs
larger than L2) and the adjoint identity <Ax, y> = <x, A^T y> is checked.

--op batched times independent scans of uneven size: --scans scans with n
drawn from {256, 384, 512, 768, 1024} and angles from {180, 360, 720, 1024,
1500} (seed 4), one slice each, seeded ellipse phantoms with 1 % Gaussian
noise, the sinogram normalised by its maximum, FBP start, prior weight
beta ~ U[0.1, 2]; --iters MBIR iterations solved once as one batched graph
(tc_mbir_batched) and once as one graph-captured solve per scan.

--op autograd times the differentiable path: forward and backward of a
10-iteration unrolled, per-iteration checkpointed reconstruction with the
gradient taken with respect to beta and sigma.

--psf random installs a random even point-spread function instead of
computing the polar one, which skips the NUFFT set-up when only the Toeplitz
or solver kernels are of interest (the operators' cost does not depend on the
values).
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np


def _events(torch, fn, reps):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _batched(a, torch, phantom, Plan):
    from .plan import BatchScan, mbir_batched
    rng = np.random.default_rng(4)
    sizes = rng.choice([256, 384, 512, 768, 1024], a.scans)
    nangs = rng.choice([180, 360, 720, 1024, 1500], a.scans)
    betas = rng.uniform(0.1, 2.0, a.scans)
    sigma = 0.05
    scans = []
    for i, (n, P) in enumerate(zip(sizes.tolist(), nangs.tolist())):
        ang = (np.arange(P) * (np.pi / P)).astype(np.float32)
        pl = Plan(n, ang, pow2_toeplitz=True)  # the batched passes take powers of two
        img = phantom.ellipse_slices(1, n, seed=100 + i)
        sino = pl.radon(img)
        sino += 0.01 * float(sino.max()) * torch.randn(sino.shape, device="cuda",
                                                      generator=torch.Generator("cuda").manual_seed(i))
        sino /= float(sino.max())
        scans.append(dict(plan=pl, aty=pl.iradon(sino), x0=pl.iradon(sino, ramp=True),
                          sino_sq=float((sino.double() ** 2).sum()), beta=float(betas[i])))
    torch.cuda.synchronize()
    K = a.iters
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # batched (one graph for all scans)
    xs = [s["x0"].clone() for s in scans]
    bs = [BatchScan(s["plan"], s["aty"], s["sino_sq"], x, sigma, 1.2, s["beta"]) for s, x in zip(scans, xs)]
    mbir_batched(bs, 2)  # warm-up
    xs = [s["x0"].clone() for s in scans]
    bs = [BatchScan(s["plan"], s["aty"], s["sino_sq"], x, sigma, 1.2, s["beta"]) for s, x in zip(scans, xs)]
    torch.cuda.synchronize()
    e0.record()
    hist = mbir_batched(bs, K)
    e1.record()
    torch.cuda.synchronize()
    t_batched = e0.elapsed_time(e1) / 1e3
    # one graph-captured solve per scan
    scans[0]["plan"].mbir_solve(scans[0]["aty"], scans[0]["sino_sq"], scans[0]["x0"], 2, sigma, 1.2,
                                scans[0]["beta"])
    torch.cuda.synchronize()
    e0.record()
    seq = [s["plan"].mbir_solve(s["aty"], s["sino_sq"], s["x0"], K, sigma, 1.2, s["beta"])
           for s in scans]
    e1.record()
    torch.cuda.synchronize()
    t_seq = e0.elapsed_time(e1) / 1e3
    diff = max(float((xb - xq).norm() / xq.norm()) for xb, (xq, _) in zip(xs, seq))
    same_attempts = all(np.array_equal(hb[:, 2], hq[:, 2]) for hb, (_, hq) in zip(hist, seq))
    for s in scans:
        s["plan"].close()
    return {"op": "batched", "scans": a.scans, "iters": K, "sizes": sizes.tolist(),
            "angles": nangs.tolist(), "slice_iters": a.scans * K,
            "batched_s": t_batched, "per_scan_s": t_seq,
            "batched_slice_iters_per_s": a.scans * K / t_batched,
            "per_scan_slice_iters_per_s": a.scans * K / t_seq,
            "speedup": t_seq / t_batched, "max_rel_diff_batched_vs_per_scan": diff,
            "same_attempts": same_attempts, "attempts": int(hist[:, :, 2].sum())}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", default="pair",
                    choices=["pair", "radon", "iradon", "toeplitz", "solve", "autograd", "batched",
                             "slab", "e2e"])
    ap.add_argument("--scans", type=int, default=48)
    ap.add_argument("--slabs", type=int, default=2, help="slabs for --op slab")
    ap.add_argument("--autotune", action="store_true",
                    help="plan created with TC_PLAN_AUTOTUNE (measured spreading tiles)")
    ap.add_argument("--n", type=int, default=1536)
    ap.add_argument("--inner", type=int, default=1024, help="phantom width embedded in n")
    ap.add_argument("--nproj", type=int, default=1500)
    ap.add_argument("--slices", type=int, default=64)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--psf", default="polar", choices=["polar", "random"])
    ap.add_argument("--plain", action="store_true", help="host-driven solve (no graph)")
    ap.add_argument("--solver-form", action="store_true",
                    help="Toeplitz as the solver applies it: H x with the FP64 x.Hx dot, no A^T y")
    a = ap.parse_args(argv)

    import torch
    from . import phantom
    from .plan import Plan

    if a.op == "batched":
        print(json.dumps(_batched(a, torch, phantom, Plan)), flush=True)
        return
    if a.op == "e2e":
        print(json.dumps(_e2e(a, torch, phantom, Plan)), flush=True)
        return

    n, P, S = a.n, a.nproj, a.slices
    ang = (np.arange(P) * (np.pi / P)).astype(np.float32)
    need_polar = a.psf == "polar" or a.op in ("pair", "radon", "iradon")
    pl = Plan(n, ang, psf=(a.psf == "polar"), autotune=a.autotune)
    if a.psf == "random":
        rng = np.random.default_rng(0)
        r = rng.standard_normal((2 * n - 1, 2 * n - 1))
        pl.set_psf(0.5 * (r + r[::-1, ::-1]) / (n * n))
    out = {"op": a.op, "n": n, "nproj": P, "slices": S, "plan": pl.info}

    inner = min(a.inner, n)
    x = torch.zeros((S, n, n), device="cuda")
    o = (n - inner) // 2
    x[:, o:o + inner, o:o + inner] = phantom.ellipse_slices(S, inner, seed=0)
    x[:, o:o + inner, o:o + inner] += 0.01 * torch.randn((S, inner, inner), device="cuda",
                                                         generator=torch.Generator("cuda").manual_seed(1))

    if need_polar and a.op in ("pair", "radon", "iradon"):
        sino = pl.radon(x)
        y = torch.randn(sino.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
        if a.op in ("pair", "radon"):
            ms = _events(torch, lambda: pl.radon(x, out=sino), a.reps)
            out["radon_ms_per_slice"] = ms / S
        if a.op in ("pair", "iradon"):
            xb = torch.empty_like(x)
            ms = _events(torch, lambda: pl.iradon(y, out=xb), a.reps)
            out["iradon_ms_per_slice"] = ms / S
        if a.op == "pair":
            ax = pl.radon(x)
            aty = pl.iradon(y)
            lhs = float((ax.double() * y.double()).sum())
            rhs = float((x.double() * aty.double()).sum())
            out["adjoint_rel"] = abs(lhs - rhs) / (float(ax.double().norm()) * float(y.double().norm()))
    if a.op in ("pair", "toeplitz"):
        g = torch.empty_like(x)
        if a.solver_form:
            ms = _events(torch, lambda: pl.toeplitz_grad(x, None, out=g, dots=True), a.reps)
        else:
            aty = torch.randn_like(x)
            ms = _events(torch, lambda: pl.toeplitz_grad(x, aty, out=g), a.reps)
        out["toeplitz_ms_per_slice"] = ms / S
    if a.op in ("solve", "slab"):
        # A^T y = H x and ||y||^2 = x.Hx: the data of the image x itself, so
        # the objective sqrt(v.Hv - 2 v.A^T y + ||y||^2) is well defined
        aty = pl.toeplitz_grad(x) * 1.0
        sino_sq = float((x.double() * aty.double()).sum())
    if a.op == "solve":
        x0 = torch.zeros_like(x)
        pl.mbir_solve(aty, sino_sq, x0, 1, 100.0, use_graph=not a.plain)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, hist = pl.mbir_solve(aty, sino_sq, x0, a.iters, 100.0, use_graph=not a.plain)
        e1.record()
        torch.cuda.synchronize()
        out["solve_ms_per_iteration"] = e0.elapsed_time(e1) / a.iters
        out["slice_iters_per_s"] = S * a.iters / (e0.elapsed_time(e1) / 1e3)
        out["attempts"] = int(hist[:, 2].sum())
    if a.op == "slab":
        # the volume as --slabs consecutive slabs in lockstep on this GPU
        # (halo copies, summed step tests, one host round trip per attempt)
        # against the whole-volume host-driven solve of the same inputs
        from .slab import Slab, solve_slabs_local
        x0 = torch.zeros_like(x)

        def timed(fn):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1), r

        bounds = np.linspace(0, S, a.slabs + 1).round().astype(int)

        def sharded(iters):
            slabs = [Slab(pl, aty[p:q].contiguous(), sino_sq, x0[p:q].contiguous(), iters, 100.0)
                     for p, q in zip(bounds[:-1], bounds[1:])]
            res = solve_slabs_local(slabs)
            for sl in slabs:
                sl.close()
            return torch.cat([r[0] for r in res]), res[0][1]

        pl.mbir_solve(aty, sino_sq, x0, 1, 100.0, use_graph=False)
        sharded(1)
        ms_w, (xw, hw) = timed(lambda: pl.mbir_solve(aty, sino_sq, x0, a.iters, 100.0, use_graph=False))
        ms_s, (xs, hs) = timed(lambda: sharded(a.iters))
        out["attempts_whole"] = int(hw[:, 2].sum())
        out["attempts_slabs"] = int(hs[:, 2].sum())
        out["slabs"] = a.slabs
        out["whole_ms_per_iteration"] = ms_w / a.iters
        out["slabs_ms_per_iteration"] = ms_s / a.iters
        out["max_rel_diff"] = float((xs - xw).norm() / xw.norm())
    if a.op == "autograd":
        from .autograd import unrolled_mbir
        aty = pl.toeplitz_grad(x) * 1.0
        x0 = 0.9 * x
        K = 10

        def fwd_bwd():
            beta = torch.tensor(0.5, dtype=torch.float64, requires_grad=True)
            sigma = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
            xk = unrolled_mbir(x0, pl, aty, K, 0.5 / pl.info["lipschitz"], beta, sigma)
            (0.5 * ((xk - x) ** 2).sum()).backward()
            return float(beta.grad), float(sigma.grad)

        ms = _events(torch, fwd_bwd, a.reps)
        out["unrolled_iters"] = K
        out["autograd_ms"] = ms
        out["autograd_ms_per_slice_iter"] = ms / (S * K)
    pl.close()
    print(json.dumps(out), flush=True)


def _e2e(a, torch, phantom, Plan):
    """cTomocam.mbir (the reference binding's call) on a pinned host sinogram
    of foam slices: --slices x --n, --nproj angles, --iters iterations; wall
    time of the call, copies and the whole mbir2 set-up included."""
    import time
    from . import cTomocam
    S, n, P = a.slices, a.n, a.nproj
    ang = (np.arange(P) * (np.pi / P)).astype(np.float32)
    vol = phantom.foam_volume(S, n, 2000, seed=0, device=torch.device("cuda", 0))
    pl = Plan(n, ang, psf=False)
    sino = phantom.transmission_noise(pl.radon(vol), 1e4, 3.0, seed=0)
    pl.close()
    host = torch.empty(sino.shape, dtype=torch.float32, pin_memory=True)
    host.copy_(sino)
    del vol, sino
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    out = cTomocam.mbir(host.numpy(), ang, (n - 1) / 2.0 + 0.5, a.iters, 100.0, 1e-4, 1e-4)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"op": "e2e", "n": n, "nproj": P, "slices": S, "iters": a.iters, "seconds": dt,
            "slice_iters_per_s": S * a.iters / dt, "finite": bool(np.isfinite(out).all())}


if __name__ == "__main__":
    main()
