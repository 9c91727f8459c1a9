"""The h5py-free HDF5 reader (tomocam_b200.h5), CPU only.

Files come from the package's own Writer (the layout libhdf5 writes by
default: superblock 0, version-1 object headers, symbol-table groups,
contiguous and B-tree-chunked datasets) and from a small generator below for
the newer layout (superblock 2, version-2 object headers, link messages,
layout 4 with single-chunk and implicit chunk indexes; checksums written as
zeros, which the reader does not verify).  The reader must return the
reference Reader's results (src/hdf5/reader.h): dims, read_sinogram
([P][S][D] -> [S][P][D] slabs), read2 and read, and refuse what it cannot
read with an H5Error.
"""
import struct

import numpy as np
import pytest

from tomocam_b200 import h5


@pytest.fixture
def sino():
    return np.random.default_rng(0).random((12, 7, 10)).astype(np.float32)


def test_contiguous_and_groups(tmp_path, sino):
    f = tmp_path / "scan.h5"
    th = np.linspace(0, np.pi, 12, endpoint=False).astype(np.float32)
    with h5.Writer(f) as w:
        w.write("/exchange/data", sino)
        w.write("/exchange/theta", th)
        w.write("/exchange/white", np.ones((2, 7, 10), np.float32))
        w.write("/meta/n", np.arange(3, dtype=np.int64))
    with h5.Reader(f) as r:
        assert r.shape("/exchange/data") == (12, 7, 10)
        assert [r.dims("/exchange/data", d) for d in range(3)] == [12, 7, 10]
        np.testing.assert_array_equal(r.read_sinogram("/exchange/data"), sino.transpose(1, 0, 2))
        np.testing.assert_array_equal(r.read_sinogram("/exchange/data", 2, 5),
                                      sino[:, 2:5].transpose(1, 0, 2))
        np.testing.assert_array_equal(r.read2("/exchange/data", 3, 7), sino[3:7])
        np.testing.assert_array_equal(r.read("/exchange/theta"), th)
        np.testing.assert_array_equal(r.read("meta/n"), [0, 1, 2])
        # a contiguous dataset is mapped, not read
        assert isinstance(r.psd("/exchange/data").base, np.memmap) or \
            isinstance(r.psd("/exchange/data"), np.memmap)


@pytest.mark.parametrize("chunks", [(12, 7, 10), (5, 3, 4), (1, 7, 10), (12, 1, 3)])
def test_chunked_btree(tmp_path, sino, chunks):
    f = tmp_path / "chunked.h5"
    with h5.Writer(f) as w:
        w.write("data", sino, chunks=chunks)
    with h5.Reader(f) as r:
        np.testing.assert_array_equal(r.psd("data"), sino)
        np.testing.assert_array_equal(r.read_sinogram("data", 1, 6), sino[:, 1:6].transpose(1, 0, 2))


def test_many_members_and_byte_orders(tmp_path):
    f = tmp_path / "many.h5"
    arrs = {f"d{i:02d}": np.full((2, 3, 4), i, np.float32) for i in range(20)}
    with h5.Writer(f) as w:
        for k, v in arrs.items():
            w.write("/g/" + k, v)
        w.write("/be", np.arange(6, dtype=">f4").reshape(1, 2, 3))
        w.write("/f8", np.arange(6, dtype="<f8").reshape(1, 2, 3))
    with h5.Reader(f) as r:
        for k, v in arrs.items():
            np.testing.assert_array_equal(r.psd("/g/" + k), v)
        np.testing.assert_array_equal(r.psd("/be", strict=False).reshape(-1), np.arange(6))
        with pytest.raises(h5.H5Error, match="mismatch"):
            r.read_sinogram("/be")
        with pytest.raises(h5.H5Error, match="mismatch"):
            r.read_sinogram("/f8")
        np.testing.assert_array_equal(r.read_sinogram("/f8", strict=False),
                                      np.arange(6, dtype=np.float32).reshape(2, 1, 3))


def test_errors(tmp_path, sino):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"not hdf5 at all" * 10)
    with pytest.raises(h5.H5Error, match="not an HDF5 file"):
        h5.Reader(bad)
    f = tmp_path / "ok.h5"
    with h5.Writer(f) as w:
        w.write("/exchange/data", sino)
        w.write("/flat", sino[0])
    with h5.Reader(f) as r:
        with pytest.raises(h5.H5Error, match="missing"):
            r.psd("/exchange/nothing")
        with pytest.raises(h5.H5Error, match="not 3D"):
            r.dims("/flat", 0)
        with pytest.raises(h5.H5Error, match="out of bounds"):
            r.read_sinogram("/exchange/data", 3, 9)


# ---------------------------------------------------------------------------
# the newer layout: superblock 2, OHDR headers, link messages, layout 4
# ---------------------------------------------------------------------------
def _ohdr2(messages):
    """Version-2 object header: (type, body) messages, 2-byte chunk size."""
    body = b"".join(struct.pack("<BHB", t, len(b), 0) + b for t, b in messages)
    return b"OHDR" + struct.pack("<BBH", 2, 0x01, len(body)) + body + b"\0\0\0\0"


def _link(name, addr):
    nb = name.encode()
    return struct.pack("<BBB", 1, 0x00, len(nb)) + nb + struct.pack("<Q", addr)


def _space2(shape):
    return struct.pack("<BBBB", 2, len(shape), 0, 1) + b"".join(struct.pack("<Q", d) for d in shape)


def _write_v2(path, a, index):
    """One dataset "/data" of float32 `a` in layout 4 (contiguous, single
    chunk or implicit 2 x 2 x 2 chunking)."""
    out = bytearray(48)
    root_at = 48
    dtm = h5._dtype_msg(np.dtype("<f4"))
    # reserve the headers, then the data
    def layout_msg(addr):
        if index == "contiguous":
            return struct.pack("<BBQQ", 4, 1, addr, a.nbytes)
        dims = a.shape if index == "single" else (2, 2, 2)
        enc = 4
        body = struct.pack("<BBBBB", 4, 2, 0, a.ndim + 1, enc)
        body += b"".join(struct.pack("<I", d) for d in dims) + struct.pack("<I", 4)
        body += struct.pack("<B", 1 if index == "single" else 2) + struct.pack("<Q", addr)
        return body
    ds_hdr_len = len(_ohdr2([(0x01, _space2(a.shape)), (0x03, dtm), (0x08, layout_msg(0))]))
    root_len = len(_ohdr2([(0x06, _link("data", 0))]))
    ds_at = root_at + root_len
    data_at = ds_at + ds_hdr_len
    if index == "implicit":
        chunks = []
        for idx in np.ndindex(*[-(-n // 2) for n in a.shape]):
            c = np.zeros((2, 2, 2), np.float32)
            sl = tuple(slice(2 * i, min(2 * i + 2, n)) for i, n in zip(idx, a.shape))
            c[tuple(slice(0, x.stop - x.start) for x in sl)] = a[sl]
            chunks.append(c.tobytes())
        payload = b"".join(chunks)
    else:
        payload = a.tobytes()
    out += _ohdr2([(0x06, _link("data", ds_at))])
    out += _ohdr2([(0x01, _space2(a.shape)), (0x03, dtm), (0x08, layout_msg(data_at))])
    out += payload
    sb = h5.SIGNATURE + struct.pack("<BBBB", 2, 8, 8, 0) + struct.pack(
        "<QQQQ", 0, h5.UNDEF, len(out), root_at) + b"\0\0\0\0"
    out[0:48] = sb
    path.write_bytes(bytes(out))


@pytest.mark.parametrize("index", ["contiguous", "single", "implicit"])
def test_newer_layout(tmp_path, index):
    a = np.random.default_rng(3).random((5, 3, 4)).astype(np.float32)
    f = tmp_path / f"v2_{index}.h5"
    _write_v2(f, a, index)
    with h5.Reader(f) as r:
        np.testing.assert_array_equal(r.psd("/data"), a)
        np.testing.assert_array_equal(r.read_sinogram("data", 1, 3), a[:, 1:3].transpose(1, 0, 2))
