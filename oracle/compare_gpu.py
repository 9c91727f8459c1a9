"""Same-GPU comparison of the product with the reference's own GPU build.

TEST INFRASTRUCTURE: the reference side is oracle/_ref/libref_gpu.so, the
reference's sources (src/*.cpp, src/gpu/*.cu) compiled for sm_100a by
`make -C oracle ref` with cuFFT and an exact-NUDFT stand-in for cuFINUFFT.
At these sizes the stand-in is too slow for the point-spread function, so
its type-1 output is staged from the product's FP64 PSF (cast to FP32, as
the reference's own float NUFFT would deliver it); nothing else on the
timed paths touches the stand-in.  Prints one JSON line per comparison:

* toeplitz -- g = H x - A^T y on S slices of n^2: the product's register-FFT
  operator against the reference's PointSpreadFunction::convolve on cuFFT
  R2C/C2R at 2n-1 in chunks of 4 slices with its per-operation allocations
  (src/toeplitz.h:134-159, src/gradient2.cpp:62), and the same convolution
  on cuFFT at M = 4096 and 2n-1 through torch.fft (cuFFT as a comparator for
  the FFT engine);
* qggmrf -- the qGGMRF gradient on S x n^2: tc_qggmrf_grad against the
  reference's qGGMRF_kernel (src/gpu/cuTV2.cu:33-93);
* iteration -- slice-iterations/s of the MBIR iteration on S slices: the
  product's graph-captured solver against the reference's Optimizer::run2
  over gradient2 + add_total_var2 + function_value2 on host arrays, the way
  mbir2 runs it (src/mbir2.cpp:114-141, PCIe transfers per operation).

    python -m oracle.compare_gpu --n 2048 --nproj 1969 --slices 256 --iter-slices 16
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


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


def _host(torch, fn, reps):
    fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) * 1e3 / reps


def _rel(a, b):
    return float((a - b).double().norm() / b.double().norm())


def _stage_psf(lib, psf64):
    k = psf64.shape[-1]
    buf = np.zeros((k, k), np.complex64)
    buf.real = psf64.reshape(k, k)
    rc = lib.ref_standin_stage(1, k, k, 1, 0, buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes)
    assert rc == 0, rc


def _torch_cufft_grad(torch, x, aty, psf64, n, M):
    """H x - aty by cuFFT (torch.fft) at size M >= 2n-1: the PSF wrapped
    circularly at offsets -(n-1)..n-1, x zero-padded, linear convolution
    cropped to the first n x n, scaled by 1/n^3 (src/toeplitz.h:134-159)."""
    k = 2 * n - 1
    pm = np.zeros((M, M), np.float64)
    idx = (np.arange(k) - (n - 1)) % M
    pm[np.ix_(idx, idx)] = psf64.reshape(k, k)
    spec = torch.fft.rfft2(torch.from_numpy(pm).to(x.device)).to(torch.complex64)
    scale = 1.0 / float(n) ** 3
    xpad = torch.zeros((4, M, M), device=x.device, dtype=torch.float32)
    out = torch.empty_like(x)

    def run():
        for s0 in range(0, x.shape[0], 4):
            b = min(4, x.shape[0] - s0)
            xpad[:b, :n, :n] = x[s0:s0 + b]
            y = torch.fft.irfft2(torch.fft.rfft2(xpad[:b]) * spec, s=(M, M))
            out[s0:s0 + b] = y[:, :n, :n] * scale - aty[s0:s0 + b]
        return out
    return run


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--nproj", type=int, default=1969)
    ap.add_argument("--slices", type=int, default=256)
    ap.add_argument("--iter-slices", type=int, default=16)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--sigma", type=float, default=100.0)
    ap.add_argument("--skip", default="", help="comma list of comparisons to skip")
    a = ap.parse_args(argv)
    skip = set(filter(None, a.skip.split(",")))

    import torch

    from tests.refbuild import gpu_lib
    from tomocam_b200.phantom import foam_volume
    from tomocam_b200.plan import Plan, qggmrf_grad

    lib = gpu_lib()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_gpu.so not built (make -C oracle ref)")
    torch.cuda.set_device(0)
    n, P, S = a.n, a.nproj, a.slices
    ang = (np.arange(P, dtype=np.float64) * (math.pi / P)).astype(np.float32)
    dev = torch.device("cuda")
    base = {"n": n, "nproj": P, "gpu": torch.cuda.get_device_name(0)}

    with Plan(n, ang) as pl:
        psf64 = pl.psf()
        _stage_psf(lib, psf64)
        h = ctypes.c_void_p()
        assert lib.ref_psf_create(ang.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), P, n, 4,
                                  ctypes.byref(h)) == 0
        lib.ref_standin_clear()
        try:
            gen = torch.Generator(device=dev).manual_seed(0)
            if "toeplitz" not in skip:
                x = torch.rand((S, n, n), device=dev, generator=gen)
                aty = torch.rand((S, n, n), device=dev, generator=gen)
                g_me = torch.empty_like(x)
                g_ref = torch.empty_like(x)
                t_me = _events(torch, lambda: pl.toeplitz_grad(x, aty, out=g_me), 5)
                t_ref = _host(torch, lambda: lib.ref_psf_grad_dev(
                    h, x.data_ptr(), aty.data_ptr(), g_ref.data_ptr(), S), 3)
                res = dict(base, comparison="toeplitz", slices=S,
                           product_ms_per_slice=t_me / S, reference_ms_per_slice=t_ref / S,
                           speedup=t_ref / t_me, rel_diff=_rel(g_me, g_ref))
                for M in sorted({4096 if n <= 2048 else 2 * n, 2 * n - 1}):
                    run = _torch_cufft_grad(torch, x, aty, psf64, n, M)
                    t_cf = _events(torch, run, 3)
                    res[f"cufft_M{M}_ms_per_slice"] = t_cf / S
                    res[f"cufft_M{M}_rel_diff"] = _rel(run(), g_me)
                print(json.dumps(res), flush=True)
                del x, aty, g_me, g_ref
            if "qggmrf" not in skip:
                x = torch.rand((S, n, n), device=dev, generator=gen)
                g1 = torch.zeros_like(x)
                g2 = torch.zeros_like(x)
                t_me = _events(torch, lambda: qggmrf_grad(x, g1, a.sigma, 1.2), 5)
                t_ref = _host(torch, lambda: lib.ref_qggmrf_dev(x.data_ptr(), g2.data_ptr(), S, n,
                                                                n, a.sigma, 1.2), 3)
                g1.zero_()
                g2.zero_()
                qggmrf_grad(x, g1, a.sigma, 1.2)
                torch.cuda.synchronize()
                lib.ref_qggmrf_dev(x.data_ptr(), g2.data_ptr(), S, n, n, a.sigma, 1.2)
                print(json.dumps(dict(base, comparison="qggmrf", slices=S,
                                      product_ms_per_slice=t_me / S,
                                      reference_ms_per_slice=t_ref / S, speedup=t_ref / t_me,
                                      rel_diff=_rel(g1, g2))), flush=True)
                del x, g1, g2
            if "iteration" not in skip:
                Si, K = a.iter_slices, a.iters
                vol = foam_volume(Si, n, seed=0)
                y = pl.radon(vol)
                aty = pl.iradon(y)
                x0 = pl.iradon(y, ramp=True)
                sino_sq = float((y.double() ** 2).sum())
                torch.cuda.synchronize()
                step = min(1.0 / float(pl.info["lipschitz"]), 1.0)
                pl.mbir_solve(aty, sino_sq, x0, K, a.sigma, step=step)   # capture + warm-up
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                x_me, _ = pl.mbir_solve(aty, sino_sq, x0, K, a.sigma, step=step)
                torch.cuda.synchronize()
                t_me = time.perf_counter() - t0
                xr = x0.cpu().numpy().copy()
                atyh = aty.cpu().numpy()
                t0 = time.perf_counter()
                rc = lib.ref_run2_host(h, xr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                       atyh.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), Si,
                                       sino_sq, a.sigma, 1.2, K, step)
                t_ref = time.perf_counter() - t0
                assert rc == 0
                diff = _rel(x_me, torch.from_numpy(xr).to(dev))
                print(json.dumps(dict(base, comparison="iteration", slices=Si, iters=K,
                                      step=step,
                                      product_slice_iters_per_s=Si * K / t_me,
                                      reference_slice_iters_per_s=Si * K / t_ref,
                                      speedup=t_ref / t_me, rel_diff=diff)), flush=True)
        finally:
            lib.ref_psf_destroy(h)


if __name__ == "__main__":
    main()
