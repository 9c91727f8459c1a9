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


if __name__ == "__main__":
    make_qggmrf_ref()
    make_operators()
    make_mbir()
    print("fixtures written to", HERE)
