"""Toeplitz gradient with a given PSF (reference tomocam/gradients.py:5-28)."""
import numpy as np

from ._ext import cTomocam


def gradients(model, sinoT, psf):
    """H model - sinoT, H the convolution with ``psf`` scaled by 1/N^3.

    model, sinoT: float32 [S, N, N]; psf: [2N-1, 2N-1] (offset index - (N-1)),
    as produced by the point-spread-function step of MBIR.
    """
    model = np.ascontiguousarray(model, dtype=np.float32)
    sinoT = np.ascontiguousarray(sinoT, dtype=np.float32)
    psf = np.ascontiguousarray(psf, dtype=np.float64)
    return cTomocam.toeplitz_gradients(model, sinoT, psf)
