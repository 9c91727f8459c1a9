"""MBIR and its building blocks, after the reference's tomocam/modeling.py:5-79."""
import numpy as np

from ._ext import cTomocam


def calc_gradients(model, sinogram, angles, center=0, over_sample=2):
    """Data gradient A^T (A model - sinogram) by NUFFT radon / back-projection.

    model [S, N, N], sinogram [S, P, N], angles [P]; float32.  Returns [S, N, N].
    (The reference documents this function but its binding was never built.)
    """
    if model.dtype != np.float32 and sinogram.dtype != np.float32 and angles.dtype != np.float32:
        raise ValueError('input data must be single precision')
    return cTomocam.gradients(model, sinogram, angles, center, over_sample)


def update_total_variation(model, gradients, smoothness=1.0E-03, p=1.2):
    """Add the qGGMRF prior gradient of ``model`` to ``gradients`` in place.

    sigma = 1 / smoothness, as MBIR maps its smoothness argument.
    """
    if model.dtype != np.float32 and gradients.dtype != np.float32:
        raise ValueError('input data must be single precision')
    if smoothness <= 0:
        raise ValueError('smoothness value must be greater than 0')
    cTomocam.total_variation(gradients, model, 1.0 / smoothness, p)
    return gradients


def MBIR(sinogram, angles, center, num_iters=100, smoothness=0.01, tol=1.0E-04, xtol=1.0E-04,
         beta=1.0):
    """Model-based iterative reconstruction (tomocam::mbir2 semantics).

    sinogram [S, P, D] float32, angles [P] radians, center of rotation in
    pixels.  Returns float32 [S, D, D].  tol and xtol are accepted and, as in
    the reference, unused.  beta multiplies the prior's gradient; the
    reference has no such parameter and corresponds to beta = 1.
    """
    if sinogram.dtype != np.float32:
        sinogram = sinogram.astype(np.float32)
    if angles.dtype != np.float32:
        angles = angles.astype(np.float32)
    if smoothness <= 0:
        raise ValueError('smoothness value must be greater than 0')
    sigma = 1. / smoothness
    if beta == 1.0:
        return cTomocam.mbir(sinogram, angles, center, num_iters, sigma, tol, xtol)
    return cTomocam.mbir(sinogram, angles, center, num_iters, sigma, tol, xtol,
                         prior_weight=float(beta))
