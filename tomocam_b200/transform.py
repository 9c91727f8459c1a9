"""radon / radon_adj with the signatures of the reference's tomocam/transform.py:4-53."""
import numpy as np

from ._ext import cTomocam


def radon(volume, angles, center=None, over_sample=1.5):
    """Radon transform of a (stack of) square image(s) by NUFFT.

    volume: float32 [S, N, N] or [N, N]; angles: float32 [P] radians.
    Returns float32 [S, P, N].  ``center`` and ``over_sample`` are accepted
    for the reference signature; the forward projection has no centre shift
    and the NUFFT upsampling is fixed at 2.
    """
    if volume.dtype != np.float32 and angles.dtype != np.float32:
        raise ValueError('input data-type must be single precision')
    return cTomocam.radon(volume, angles, center, over_sample)


def radon_adj(sinogram, angles, center, over_sample=1.5):
    """Back-projection (adjoint radon) of a sinogram [S, P, D] about ``center``.

    Pads and centres the detector as the reference's backproject binding
    does (src/pyTomocam.cpp:94-114) and returns float32 [S, D, D].
    """
    if sinogram.dtype != np.float32 and angles.dtype != np.float32:
        raise ValueError('input data-type must be single precision')
    return cTomocam.radon_adj(sinogram, angles, center, over_sample)
