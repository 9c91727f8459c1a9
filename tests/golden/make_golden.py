"""Generate the committed golden fixtures in tests/golden/.

Run in a container that has the reference tree (it reads nothing from it at
test time):

    make -C oracle ref            # compiles the reference's CPU qGGMRF
    python tests/golden/make_golden.py

* qggmrf_ref.npz -- input drawn from the reference test's own random stream
  (test/timer.h NPRandom, mt19937 seed 5489) and the outputs of the
  reference's cpuTotalVar (test/tvd.cpp:40-75) for three (sigma, p) pairs.
  These pin both the oracle's prior and the CUDA stencil to the reference's
  code.
* operators_n32.npz -- FP64 oracle outputs (exact non-uniform DFT) of radon,
  back-projection (plain and ramp-filtered), the PSF and the Toeplitz
  gradient on a 32 x 32 ellipse phantom with 24 angles, so the GPU tests
  compare against fixed numbers as well as the live oracle.
* mbir_n24.npz -- FP64 oracle run of tomocam::mbir2 semantics: 2 slices of a
  24-pixel-detector sinogram, 30 angles, centre 11.7, 6 iterations.
* run2_ref.npz -- the reference's own Optimizer::run2 (src/optimize.h:96-154,
  compiled into oracle/_ref/libref_run2.so) driven by the FP64 oracle's
  gradient (gradient2 + qGGMRF) and objective (sqrt function_value2), for a
  plain case and a backtracking case: inputs, the reference's result, its
  gradient-evaluation count and every objective value it asked for.  These
  pin oracle.run2's control flow to the reference's code.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def make_qggmrf_ref():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_tvd.so"))
    fp = ctypes.POINTER(ctypes.c_float)
    lib.ref_cpu_total_var.argtypes = [fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_float]
    lib.ref_nprandom_fill.argtypes = [fp, ctypes.c_long]
    S, R, C = 4, 17, 23
    x = np.empty(S * R * C, np.float32)
    lib.ref_nprandom_fill(x.ctypes.data_as(fp), x.size)
    x = x.reshape(S, R, C)
    params = np.array([[10.0, 1.2], [0.5, 1.2], [0.05, 1.5]], dtype=np.float32)
    outs = []
    for sigma, p in params:
        o = np.empty_like(x)
        rc = lib.ref_cpu_total_var(x.ctypes.data_as(fp), o.ctypes.data_as(fp), S, R, C,
                                   float(sigma), float(p))
        assert rc == 0
        outs.append(o)
    np.savez_compressed(os.path.join(HERE, "qggmrf_ref.npz"), x=x, params=params,
                        out=np.stack(outs))


def make_operators():
    n, P = 32, 24
    ang = O.uniform_angles(P).astype(np.float32)
    a64 = ang.astype(np.float64)
    x = O.ellipse_phantom(n, 10, 3)[None].astype(np.float32)
    rng = np.random.default_rng(21)
    sino = rng.standard_normal((1, P, n)).astype(np.float32)
    aty = rng.standard_normal((1, n, n)).astype(np.float32)
    psf = O.psf_kernel(n, a64)
    np.savez_compressed(
        os.path.join(HERE, "operators_n32.npz"), angles=ang, x=x, sino=sino, aty=aty,
        radon=O.project(x.astype(np.float64), a64),
        backproject=O.backproject(sino.astype(np.float64), a64),
        fbp=O.backproject(sino.astype(np.float64), a64, fbp=True),
        psf=psf, toeplitz_grad=O.gradient2(x.astype(np.float64), aty.astype(np.float64), psf))


def make_mbir():
    D, P = 24, 30
    ang = O.uniform_angles(P).astype(np.float32)
    img = np.stack([O.ellipse_phantom(D, 6, 40 + s) for s in range(2)])
    sino = O.project(img, ang.astype(np.float64)).astype(np.float32)
    rec = O.Run2Record()
    out = O.mbir2(sino, ang.astype(np.float64), 11.7, 6, sigma=20.0, record=rec)
    np.savez_compressed(os.path.join(HERE, "mbir_n24.npz"), angles=ang, sino=sino, center=11.7,
                        num_iters=6, sigma=20.0, out=out,
                        history=np.array([[e, xe] for _, e, xe in rec.iters]))


def run2_cases():
    """The two solver cases of run2_ref.npz (inputs only, FP64)."""
    cases = {}
    for name, n, P, S, seed, scale, step_mul, weight, sigma, iters in (
            ("plain", 16, 20, 2, 7, 1.0, 1.0, 1.0, 5.0, 6),
            ("backtrack", 16, 20, 2, 3, 1e-4, 2.5, 1e-3, 1.0, 5)):
        ang = O.uniform_angles(P)
        img = np.stack([O.ellipse_phantom(n, 6, seed + s) for s in range(S)])
        sino = O.project(img, ang)
        sino = sino + 0.01 * sino.max() * np.random.default_rng(seed).standard_normal(sino.shape)
        sino = sino * scale
        aty = O.backproject(sino, ang)
        x0 = O.backproject(sino, ang, fbp=True)
        psf = O.psf_kernel(n, ang)
        step, _ = O.lipschitz_step(psf, n)
        cases[name] = dict(x0=x0, aty=aty, psf=psf, sino_sq=float(np.sum(sino ** 2)),
                           sigma=sigma, p=1.2, weight=weight, step=step * step_mul, iters=iters)
    return cases


def run2_callbacks(c):
    import math

    def grad_fn(v):
        return O.gradient2(v, c["aty"], c["psf"]) + O.qggmrf_grad(v, c["sigma"], c["p"],
                                                                  c["weight"])

    def err_fn(v):
        return math.sqrt(O.function_value2(v, c["aty"], c["psf"], c["sino_sq"]))
    return grad_fn, err_fn


def make_run2_ref():
    from tests.refbuild import ref_run2
    out = {}
    for name, c in run2_cases().items():
        g, e = run2_callbacks(c)
        res = ref_run2(c["x0"], c["iters"], c["step"], g, e)
        assert res is not None, "oracle/_ref/libref_run2.so not built (make -C oracle ref)"
        x, attempts, errs = res
        for k, v in c.items():
            out[f"{name}_{k}"] = np.asarray(v)
        out[f"{name}_out"] = x
        out[f"{name}_attempts"] = np.asarray(attempts)
        out[f"{name}_errs"] = errs
    np.savez_compressed(os.path.join(HERE, "run2_ref.npz"), **out)


if __name__ == "__main__":
    make_qggmrf_ref()
    make_operators()
    make_mbir()
    make_run2_ref()
    print("fixtures written to", HERE)
