"""Sinogram ingest from the HDF5 file layout.

The reference reads tomography datasets stored projection-major,
``[projections][slices][detector]``, and transposes them to the slice-major
``[slices][projections][detector]`` its operators use, on the host
(``src/hdf5/reader.h:67-122``).  ``sinogram_from_psd`` takes such an array
(however it was read: h5py, a memory map, a raw file) and copies a slab of
slices straight into device memory in the operators' layout with one strided
copy per projection (``tc_sino_ingest_psd``): pinned host memory is copied
directly, pageable memory through the library's pinned staging buffers.
``tomocam_b200.h5.Reader.sinogram_to_device`` reads the files themselves
(without libhdf5 or h5py) and feeds a contiguous dataset's memory map
straight to this copy.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .plan import _check_tensor, _ptr


def sinogram_from_psd(host, s0: int = 0, ns: int | None = None, out=None):
    """Slices ``s0 .. s0+ns-1`` of a host array ``host [P][S][D]`` (float32,
    C order; a numpy array or a CPU tensor, pinned or not) as a CUDA tensor
    ``[ns][P][D]``.  ``out`` (optional) receives the result."""
    if isinstance(host, torch.Tensor):
        if host.is_cuda:
            raise TypeError("host must be a host array (numpy or a CPU tensor)")
        if host.dtype != torch.float32 or not host.is_contiguous():
            host = host.to(torch.float32).contiguous()
        keep = host
        shape = tuple(host.shape)
        hptr = ctypes.cast(ctypes.c_void_p(host.data_ptr()), ctypes.POINTER(ctypes.c_float))
    else:
        keep = np.ascontiguousarray(host, dtype=np.float32)
        shape = keep.shape
        hptr = keep.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    if len(shape) != 3:
        raise ValueError(f"host must be [projections][slices][detector], got shape {shape}")
    P, S, D = (int(v) for v in shape)
    s0 = int(s0)
    ns = S - s0 if ns is None else int(ns)
    if s0 < 0 or ns < 0 or s0 + ns > S:
        raise ValueError(f"slices {s0} .. {s0 + ns - 1} are outside the {S} slices of the sinogram")
    if out is None:
        out = torch.empty((max(ns, 0), P, D), dtype=torch.float32, device="cuda")
    _check_tensor(out, (max(ns, 0), P, D), "out")
    # the copy completes before the call returns; it is ordered after the
    # work already queued on the device
    torch.cuda.current_stream().synchronize()
    _lib.call("tc_sino_ingest_psd", hptr, P, S, D, s0, ns, _ptr(out))
    del keep
    return out
