"""Generate golden fixtures from the reference's own GPU build (needs a GPU).

The reference's sources are compiled by `make -C oracle ref` into
oracle/_ref/ (libref_gpu.so with an exact-NUDFT stand-in for cuFINUFFT, and
the reference's Python module cTomocam).  This script runs them and writes:

* refgpu_prep.npz -- preproc (src/preproc.cpp:74-102) on sinograms of several
  widths and centres, postproc (src/postproc.cpp:70-97), the host pad2d
  (src/padding.cpp) and gpu::roll (src/gpu/fftshift.cu:30-40): inputs and
  the reference's outputs, bit for bit.
* refgpu_module.npz -- the reference module's radon, backproject (with
  preproc/postproc) and mbir (mbir2 end to end) on small seeded inputs.

    python tests/golden/make_golden_refgpu.py [outdir]

The CPU tests (tests/test_oracle_refgpu.py) hold the oracle to these.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from tests.refbuild import fptr, gpu_lib, ref_module  # noqa: E402

PREPROC = [(24, 11.7), (24, 12.5), (25, 12.0), (25, 11.5), (40, 17.4), (40, 23.5), (31, 3.0),
           (64, 32.0), (17, 8.49), (256, 128.0), (256, 120.6)]
POSTPROC = [(34, 24), (35, 25), (90, 64), (57, 40)]
PAD2D = [(24, 10), (25, 11), (64, 26), (40, 16)]
ROLL = [(24, 3), (24, -5), (25, 12), (25, -13), (31, 0)]


def _ip(a):
    import ctypes
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def make_prep(lib, out):
    d = {}
    for k, (D, c) in enumerate(PREPROC):
        s = np.random.default_rng(100 + k).standard_normal((2, 5, D)).astype(np.float32)
        buf = np.empty(2 * 5 * (3 * D + 8), np.float32)
        cols = np.zeros(1, np.int32)
        assert lib.ref_preproc(fptr(s), 2, 5, D, float(c), fptr(buf), buf.size, _ip(cols)) == 0
        m = int(cols[0])
        d[f"pre{k}_in"], d[f"pre{k}_center"] = s, np.float32(c)
        d[f"pre{k}_out"] = buf[:2 * 5 * m].reshape(2, 5, m).copy()
    for k, (n, npix) in enumerate(POSTPROC):
        x = np.random.default_rng(200 + k).standard_normal((2, n, n)).astype(np.float32)
        buf = np.empty(x.size, np.float32)
        m = np.zeros(1, np.int32)
        assert lib.ref_postproc(fptr(x), 2, n, npix, fptr(buf), buf.size, _ip(m)) == 0
        q = int(m[0])
        d[f"post{k}_in"], d[f"post{k}_npix"] = x, np.int32(npix)
        d[f"post{k}_out"] = buf[:2 * q * q].reshape(2, q, q).copy()
    for k, (n, npad) in enumerate(PAD2D):
        x = np.random.default_rng(300 + k).standard_normal((2, n, n)).astype(np.float32)
        q = n + npad
        buf = np.empty(2 * q * q, np.float32)
        m = np.zeros(1, np.int32)
        assert lib.ref_pad2d(fptr(x), 2, n, npad, 0, fptr(buf), buf.size, _ip(m)) == 0
        d[f"pad{k}_in"], d[f"pad{k}_npad"] = x, np.int32(npad)
        d[f"pad{k}_out"] = buf.reshape(2, q, q).copy()
    for k, (C, delta) in enumerate(ROLL):
        x = np.random.default_rng(400 + k).standard_normal((2, 3, C)).astype(np.float32)
        o = np.empty_like(x)
        assert lib.ref_roll(fptr(x), fptr(o), 2, 3, C, delta) == 0
        d[f"roll{k}_in"], d[f"roll{k}_delta"], d[f"roll{k}_out"] = x, np.int32(delta), o
    np.savez_compressed(os.path.join(out, "refgpu_prep.npz"), **d)


def make_module(mod, out):
    d = {}
    n, P = 32, 24
    ang = O.uniform_angles(P).astype(np.float32)
    img = np.stack([O.ellipse_phantom(n, 8, 500 + s) for s in range(2)]).astype(np.float32)
    d["radon_angles"], d["radon_in"] = ang, img
    d["radon_out"] = mod.radon(img, ang)
    D, P2, c = 40, 31, 17.4
    ang2 = O.uniform_angles(P2).astype(np.float32)
    sino = np.random.default_rng(600).standard_normal((2, P2, D)).astype(np.float32)
    d["bp_angles"], d["bp_in"], d["bp_center"] = ang2, sino, np.float32(c)
    d["bp_out"] = mod.backproject(sino, ang2, c)
    D, P3, S, iters, sigma = 80, 60, 2, 8, 5.0
    ang3 = O.uniform_angles(P3).astype(np.float32)
    img3 = np.stack([O.ellipse_phantom(D, 10, 11 + s) for s in range(S)])
    s3 = O.project(img3, ang3.astype(np.float64))
    s3 = (s3 + 0.01 * s3.max() * np.random.default_rng(11).standard_normal(s3.shape))
    s3 = s3.astype(np.float32)
    cen = D / 2 - 0.3
    d["mbir_angles"], d["mbir_in"], d["mbir_center"] = ang3, s3, np.float32(cen)
    d["mbir_iters"], d["mbir_sigma"] = np.int32(iters), np.float32(sigma)
    d["mbir_out"] = mod.mbir(s3, ang3, cen, iters, sigma, 1e-4, 1e-4)
    np.savez_compressed(os.path.join(out, "refgpu_module.npz"), **d)


if __name__ == "__main__":
    out = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out, exist_ok=True)
    lib = gpu_lib()
    mod = ref_module()
    assert lib is not None and mod is not None, "run `make -C oracle ref` first"
    make_prep(lib, out)
    make_module(mod, out)
    print("fixtures written to", out)
