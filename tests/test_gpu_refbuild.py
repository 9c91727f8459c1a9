"""The product against the reference's own GPU build, on the same B200.

`make -C oracle ref` compiles the reference's sources (src/*.cpp,
src/gpu/*.cu for sm_100a, cuFFT) and its Python module cTomocam
(src/pyTomocam.cpp) into oracle/_ref/, with cuFINUFFT -- absent from this
image -- replaced by an exact non-uniform DFT that implements the cuFINUFFT
entry points the reference calls (oracle/refgpu/).  Everything else on the
reference path runs unchanged: preproc/postproc/pad2d and their kernels,
the PointSpreadFunction on cuFFT, the qGGMRF kernel, gradient2,
function_value2 and Optimizer::run2 inside mbir2.

Tolerances: pre/post-processing is data movement and must match bit for
bit; operators 1e-5 against the FP64 oracle for both builds; whole
reconstructions 1e-4 between the builds (both are FP32; the reference forms
its k-space points in FP32, which at these sizes moves results by ~1e-6).
The tests skip when oracle/_ref was not built.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import phantom_stack, rel_l2
from tests.refbuild import fptr, gpu_lib, ref_module

pytestmark = pytest.mark.gpu

TOL_OP = 1e-5
TOL_RECON = 1e-4


@pytest.fixture(scope="module")
def ref():
    lib = gpu_lib()
    if lib is None:
        pytest.skip("reference GPU build not compiled (make -C oracle ref)")
    return lib


def _preproc_ref(lib, sino, center):
    S, P, D = sino.shape
    cap = S * P * (3 * D + 8)
    out = np.empty(cap, np.float32)
    cols = np.zeros(1, np.int32)
    assert lib.ref_preproc(fptr(sino), S, P, D, float(center), fptr(out), cap, _ip(cols)) == 0
    return out[:S * P * int(cols[0])].reshape(S, P, int(cols[0]))


def _ip(a):
    import ctypes
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


# centres on both sides of the detector middle, half-integers (std::round
# rounds them away from zero), and one offset larger than the default padding
PREPROC_CASES = [(24, 11.7), (24, 12.5), (25, 12.0), (25, 11.5), (40, 17.4), (40, 23.5),
                 (31, 3.0), (64, 32.0), (17, 8.49)]


@pytest.mark.parametrize("D,center", PREPROC_CASES)
def test_preproc_oracle_matches_reference(ref, D, center):
    sino = np.random.default_rng(D).standard_normal((2, 7, D)).astype(np.float32)
    out = _preproc_ref(ref, sino, center)
    mine = O.preproc(sino.astype(np.float64), center)
    assert out.shape == mine.shape
    assert np.array_equal(out, mine.astype(np.float32))


@pytest.mark.parametrize("n,npix", [(34, 24), (35, 25), (362, 256), (57, 40)])
def test_postproc_oracle_matches_reference(ref, n, npix):
    x = np.random.default_rng(n).standard_normal((2, n, n)).astype(np.float32)
    out = np.empty(x.size, np.float32)
    m = np.zeros(1, np.int32)
    assert ref.ref_postproc(fptr(x), 2, n, npix, fptr(out), out.size, _ip(m)) == 0
    k = int(m[0])
    got = out[:2 * k * k].reshape(2, k, k)
    mine = O.postproc(x.astype(np.float64), npix)
    assert got.shape == mine.shape
    assert np.array_equal(got, mine.astype(np.float32))


@pytest.mark.parametrize("n,npad", [(24, 10), (25, 11), (256, 106), (40, 16)])
def test_pad2d_oracle_matches_reference(ref, n, npad):
    x = np.random.default_rng(npad).standard_normal((2, n, n)).astype(np.float32)
    k = n + npad
    out = np.empty(2 * k * k, np.float32)
    m = np.zeros(1, np.int32)
    assert ref.ref_pad2d(fptr(x), 2, n, npad, 0, fptr(out), out.size, _ip(m)) == 0
    assert int(m[0]) == k
    got = out.reshape(2, k, k)
    mine = O.pad2d_symmetric(x.astype(np.float64), npad)
    assert np.array_equal(got, mine.astype(np.float32))


@pytest.mark.parametrize("C,delta", [(24, 3), (24, -5), (25, 12), (25, -13), (31, 0)])
def test_roll_matches_numpy_semantics(ref, C, delta):
    """gpu::roll (src/gpu/fftshift.cu:30-40): out[k] = in[(k + delta) mod C]."""
    x = np.random.default_rng(C).standard_normal((2, 3, C)).astype(np.float32)
    out = np.empty_like(x)
    assert ref.ref_roll(fptr(x), fptr(out), 2, 3, C, delta) == 0
    assert np.array_equal(out, np.roll(x, -delta, axis=-1))


# The reference's qGGMRF kernel (src/gpu/cuTV2.cu:33-76) and its dot kernel
# (src/gpu/gpu_ops.cu:230-249) place __syncthreads() inside a bounds branch;
# the checker runs them only on sizes whose every thread block is full
# (rows and columns multiples of 16, dot lengths multiples of 256).
@pytest.mark.parametrize("S,R,C,sigma,p", [(4, 16, 16, 2.0, 1.2), (3, 32, 48, 0.5, 1.2),
                                           (1, 48, 32, 5.0, 1.5), (6, 64, 64, 100.0, 1.2)])
def test_qggmrf_kernel_matches_reference_kernel(ref, S, R, C, sigma, p):
    import torch
    from tomocam_b200.plan import qggmrf_grad
    assert R % 16 == 0 and C % 16 == 0
    rng = np.random.default_rng(S * R + C)
    x = rng.random((S, R, C)).astype(np.float32)
    g0 = rng.standard_normal((S, R, C)).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    g_ref = torch.from_numpy(g0).cuda()
    g_mine = g_ref.clone()
    torch.cuda.synchronize()
    assert ref.ref_qggmrf_dev(dx.data_ptr(), g_ref.data_ptr(), S, R, C, sigma, p) == 0
    qggmrf_grad(dx, g_mine, sigma, p)
    torch.cuda.synchronize()
    prior = O.qggmrf_grad(x.astype(np.float64), sigma, p)
    d_ref = g_ref.cpu().numpy().astype(np.float64) - g0
    d_mine = g_mine.cpu().numpy().astype(np.float64) - g0
    # both kernels compute in FP32; at sigma = 100 the 26 terms of a voxel's
    # sum largely cancel and both sit about 1e-5 from the FP64 oracle while
    # agreeing with each other to a few 1e-6
    assert rel_l2(d_ref, prior) < 3e-5
    assert rel_l2(d_mine, prior) < 3e-5
    assert rel_l2(d_mine, d_ref) < 4e-6


def _psf_handle(lib, ang, n, batch):
    import ctypes
    h = ctypes.c_void_p()
    assert lib.ref_psf_create(fptr(ang), ang.size, n, batch, ctypes.byref(h)) == 0
    return h


@pytest.mark.parametrize("n,P,S", [(16, 20, 4), (33, 24, 5), (48, 40, 4)])
def test_toeplitz_gradient_matches_reference_psf_on_cufft(ref, n, P, S):
    """g = H x - A^T y: the reference's PointSpreadFunction (its own PSF
    constructor over the exact type-1 transform, R2C/C2R on cuFFT at 2n-1,
    src/toeplitz.h:51-159) against the product's register-FFT operator."""
    import torch
    from tomocam_b200.plan import Plan
    ang = O.uniform_angles(P).astype(np.float32)
    x = phantom_stack(S, n, seed=n)
    aty = np.random.default_rng(P).standard_normal((S, n, n)).astype(np.float32)
    h = _psf_handle(ref, ang, n, 4)
    try:
        dx = torch.from_numpy(x).cuda()
        da = torch.from_numpy(aty).cuda()
        g_ref = torch.empty_like(dx)
        torch.cuda.synchronize()
        assert ref.ref_psf_grad_dev(h, dx.data_ptr(), da.data_ptr(), g_ref.data_ptr(), S) == 0
    finally:
        ref.ref_psf_destroy(h)
    with Plan(n, ang) as pl:
        g_mine = pl.toeplitz_grad(dx, da)
        torch.cuda.synchronize()
    want = O.gradient2(x.astype(np.float64), aty.astype(np.float64),
                       O.psf_kernel(n, ang.astype(np.float64)))
    assert rel_l2(g_ref.cpu().numpy(), want) < TOL_OP
    assert rel_l2(g_mine.cpu().numpy(), want) < TOL_OP
    assert rel_l2(g_mine.cpu().numpy(), g_ref.cpu().numpy()) < 2 * TOL_OP


@pytest.fixture(scope="module")
def refmod(ref):
    mod = ref_module()
    if mod is None:
        pytest.skip("reference cTomocam module not compiled (make -C oracle ref)")
    return mod


@pytest.mark.parametrize("n,P", [(32, 24), (33, 30), (64, 45)])
def test_radon_matches_reference_module(refmod, n, P):
    from tomocam_b200 import cTomocam
    ang = O.uniform_angles(P).astype(np.float32)
    img = phantom_stack(2, n, seed=P)
    out_ref = refmod.radon(img, ang)
    out = cTomocam.radon(img, ang)
    want = O.project(img.astype(np.float64), ang.astype(np.float64))
    assert out.shape == out_ref.shape == want.shape
    assert rel_l2(out_ref, want) < TOL_OP
    assert rel_l2(out, out_ref) < 2 * TOL_OP


@pytest.mark.parametrize("D,P,center", [(40, 31, 20.0), (40, 31, 17.4), (33, 24, 16.5),
                                        (64, 45, 30.2)])
def test_backproject_matches_reference_module(refmod, D, P, center):
    """cTomocam.backproject = preproc, back-projection, postproc
    (src/pyTomocam.cpp:94-114), end to end through both builds."""
    from tomocam_b200 import cTomocam
    ang = O.uniform_angles(P).astype(np.float32)
    sino = np.random.default_rng(D + P).standard_normal((2, P, D)).astype(np.float32)
    out_ref = refmod.backproject(sino, ang, center)
    out = cTomocam.backproject(sino, ang, center)
    assert out.shape == out_ref.shape == (2, D, D)
    assert rel_l2(out, out_ref) < 2 * TOL_OP


def test_mbir_matches_reference_module(refmod):
    """cTomocam.mbir (src/pyTomocam.cpp:116-134 -> mbir2): normalisation, FBP
    guess, preproc, symmetric pad, A^T y, PSF, Lipschitz step, run2 over
    gradient2 + qGGMRF and function_value2, postproc -- the whole reference
    path on the GPU against the product's.  D = 80 pads to a 112-pixel grid
    (every qGGMRF and dot block full)."""
    from tomocam_b200 import cTomocam
    D, P, S, iters, sigma = 80, 60, 2, 8, 5.0
    ang = O.uniform_angles(P).astype(np.float32)
    img = phantom_stack(S, D, seed=11)
    sino = O.project(img.astype(np.float64), ang.astype(np.float64))
    sino = (sino + 0.01 * sino.max() * np.random.default_rng(11).standard_normal(sino.shape))
    sino = sino.astype(np.float32)
    center = D / 2 - 0.3
    out_ref = refmod.mbir(sino, ang, center, iters, sigma, 1e-4, 1e-4)
    out = cTomocam.mbir(sino, ang, center, iters, sigma, 1e-4, 1e-4)
    assert out.shape == out_ref.shape == (S, D, D)
    assert np.isfinite(out_ref).all()
    assert rel_l2(out, out_ref) < TOL_RECON
