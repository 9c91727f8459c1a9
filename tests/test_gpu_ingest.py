"""Sinogram ingest from the HDF5 layout ([P][S][D] -> [S][P][D] on the
device, src/hdf5/reader.h:67-122): exact against numpy's transpose, for
pageable and pinned sources, whole volumes and slabs, and a source larger
than the staging buffers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ref(a, s0, ns):
    return np.ascontiguousarray(np.transpose(a, (1, 0, 2))[s0:s0 + ns])


@pytest.mark.parametrize("P,S,D,s0,ns", [(7, 5, 9, 0, 5), (7, 5, 9, 1, 3), (300, 64, 1024, 0, 64),
                                          (300, 64, 1024, 17, 30), (5, 1, 3, 0, 1)])
def test_ingest_pageable(P, S, D, s0, ns):
    from tomocam_b200.ingest import sinogram_from_psd
    a = np.random.default_rng(P + S + D).standard_normal((P, S, D)).astype(np.float32)
    out = sinogram_from_psd(a, s0, ns).cpu().numpy()
    assert np.array_equal(out, _ref(a, s0, ns))


@pytest.mark.parametrize("s0,ns", [(0, 40), (9, 13)])
def test_ingest_pinned(s0, ns):
    import torch
    from tomocam_b200.ingest import sinogram_from_psd
    a = np.random.default_rng(5).standard_normal((120, 40, 512)).astype(np.float32)
    t = torch.from_numpy(a).pin_memory()
    out = sinogram_from_psd(t, s0, ns).cpu().numpy()
    assert np.array_equal(out, _ref(a, s0, ns))


def test_ingest_feeds_operators():
    """The ingested slab is what the operators take: back-projecting it equals
    back-projecting numpy's transpose."""
    import torch
    from oracle import oracle as O
    from tomocam_b200.ingest import sinogram_from_psd
    from tomocam_b200.plan import Plan
    n, P = 64, 45
    ang = O.uniform_angles(P).astype(np.float32)
    a = np.random.default_rng(2).standard_normal((P, 6, n)).astype(np.float32)
    with Plan(n, ang, psf=False) as pl:
        b1 = pl.iradon(sinogram_from_psd(a, 2, 3)).cpu().numpy()
        b2 = pl.iradon(torch.from_numpy(_ref(a, 2, 3)).cuda()).cpu().numpy()
    assert np.array_equal(b1, b2)


@pytest.mark.parametrize("chunks", [None, (4, 3, 8)])
def test_hdf5_file_straight_to_device(tmp_path, chunks):
    """An HDF5 [P][S][D] dataset (contiguous: memory-mapped; chunked: assembled
    on the host) into HBM as [S][P][D] slabs, src/hdf5/reader.h:67-122."""
    import torch
    from tomocam_b200 import h5
    rng = np.random.default_rng(11)
    P, S, D = 9, 6, 20
    a = rng.standard_normal((P, S, D)).astype(np.float32)
    f = tmp_path / "scan.h5"
    with h5.Writer(f) as w:
        w.write("/exchange/data", a, chunks=chunks)
    with h5.Reader(f) as r:
        full = r.sinogram_to_device("/exchange/data")
        slab = r.sinogram_to_device("/exchange/data", 2, 5)
        torch.cuda.synchronize()
    np.testing.assert_array_equal(full.cpu().numpy(), a.transpose(1, 0, 2))
    np.testing.assert_array_equal(slab.cpu().numpy(), a[:, 2:5].transpose(1, 0, 2))
