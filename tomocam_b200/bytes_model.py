"""Algorithmic HBM bytes of the hot-path operators (per slice).

The roofline figures divide these byte counts by measured kernel time.  They
count the traffic the algorithm cannot avoid with the three-pass Toeplitz
scheme and the fused stencil, not what a particular kernel happens to move
(ncu's dram__bytes_* give the latter).  float32 = 4 B, complex64 = 8 B.
"""
from __future__ import annotations


def toeplitz(n: int, m: int, slices_per_psf_read: float = 1.0, with_aty: bool = True) -> float:
    """g = H x - A^T y (or H x with the x.Hx dot) on an m x m padded grid.

    Pass 1 reads x (4 n^2) and writes the row spectra of the n image rows
    (half of a pair's n x m complex workspace: 4 n m per slice); pass 2
    reads and writes them (8 n m) and reads the m x m float PSF spectrum
    once per ``slices_per_psf_read`` slices; pass 3 reads the workspace
    (4 n m), reads A^T y or x for the dot (4 n^2) and writes g (4 n^2).
    With m = 2n this is 44 n^2 plus the PSF share.
    """
    del with_aty  # A^T y and the dot's x are the same size
    return 12.0 * n * n + 16.0 * n * m + 4.0 * m * m / max(slices_per_psf_read, 1.0)


def compulsory(n: int) -> float:
    """Bytes no Toeplitz scheme can avoid: read x and A^T y, write g."""
    return 12.0 * n * n


def update(n: int, tile_y: int = 32, tile_x: int = 64, same: bool = True) -> float:
    """Fused stencil + Nesterov update of one slice (k_mbir_update).

    Every attempt after an accepted step has x = sol (``same``): it reads sol
    (with the one-voxel tile ring re-read by the neighbouring tiles), H sol
    and A^T y, and writes the new iterate.  After a rejected step it also
    reads x (with the ring) and H x.
    """
    ring = (tile_y + 2) * (tile_x + 2) / (tile_y * tile_x)
    if same:
        return 4.0 * n * n * (ring + 3)
    return 4.0 * n * n * (2 * ring + 4)


def iteration(n: int, m: int, slices_per_psf_read: float = 1.0, same: bool = True) -> float:
    """One accepted MBIR attempt per slice: the update plus one Toeplitz apply."""
    return update(n, same=same) + toeplitz(n, m, slices_per_psf_read)


def radon(n: int, nproj: int, ndet: int) -> float:
    """Forward projection (sigma = 2 fine grid of 2n): deconvolve/pad/row FFT,
    column FFT, interpolation reading the fine grid once, detector FFT."""
    return 100.0 * n * n + 4.0 * nproj * ndet


def iradon(n: int, nproj: int, ndet: int) -> float:
    """Back-projection mirrors the forward projection."""
    return radon(n, nproj, ndet)
