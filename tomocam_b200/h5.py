"""Reading (and writing) the HDF5 files tomography data come in, without
libhdf5 or h5py.

The reference reads its sinograms with libhdf5 (``src/hdf5/reader.h``:
``Reader::dims``, ``read_sinogram`` -- a ``[projections][slices][detector]``
dataset transposed on the host to ``[slices][projections][detector]`` --,
``read2`` and ``read`` for the angles) and writes results with
``src/hdf5/writer.h``.  This module parses the file format itself (the HDF
Group's published "HDF5 File Format Specification", version 3) for the
datasets those calls handle:

* superblock versions 0 - 3;
* object headers version 1 and 2 (with continuation blocks);
* groups stored as symbol tables (v1 B-tree, local heap, symbol nodes) or as
  compact link messages; dense (fractal-heap) groups are refused;
* simple dataspaces; IEEE float32 / float64 and integer datatypes, either
  byte order;
* data layout versions 3 and 4: contiguous, and chunked without filters with
  a version-1 B-tree, single-chunk or implicit index (other indexes and any
  filter -- compression -- are refused with a clear error).

Contiguous datasets are memory-mapped, so a slab of slices reaches the device
(``Reader.sinogram_to_device``, ``tc_sino_ingest_psd``) without a host-side
transpose or a full read.  ``Writer`` produces files of the layout libhdf5
writes by default (superblock 0, version-1 object headers, symbol-table
groups, contiguous or chunked datasets); the tests read such files back.
"""
from __future__ import annotations

import os
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


class H5Error(RuntimeError):
    """The file is not HDF5, or uses a feature this reader does not handle."""


# ---------------------------------------------------------------------------
# reading
# ---------------------------------------------------------------------------
class _Buf:
    """Little-endian field reader over the mapped file."""

    def __init__(self, mm, so=8, sl=8):
        self.mm = mm
        self.so = so  # size of offsets
        self.sl = sl  # size of lengths

    def u(self, pos, n):
        return int.from_bytes(self.mm[pos:pos + n], "little")

    def off(self, pos):
        return self.u(pos, self.so)

    def ln(self, pos):
        return self.u(pos, self.sl)

    def sig(self, pos, s):
        if bytes(self.mm[pos:pos + len(s)]) != s:
            raise H5Error(f"expected {s!r} at offset {pos}")


class _Dataset:
    def __init__(self, shape, dtype, layout, addr, size, chunk, index, index_addr, filters):
        self.shape = shape
        self.dtype = dtype
        self.layout = layout          # "contiguous" | "chunked" | "compact"
        self.addr = addr
        self.size = size
        self.chunk = chunk            # chunk dims (chunked)
        self.index = index            # "btree1" | "single" | "implicit"
        self.index_addr = index_addr
        self.filters = filters


class Reader:
    """Open an HDF5 file for reading (``src/hdf5/reader.h`` ``Reader``)."""

    def __init__(self, filename):
        self.filename = os.fspath(filename)
        self._mm = np.memmap(self.filename, dtype=np.uint8, mode="r")
        mm = self._mm
        base = None
        for cand in (0, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536):
            if cand + 8 <= mm.size and bytes(mm[cand:cand + 8]) == SIGNATURE:
                base = cand
                break
        if base is None:
            raise H5Error(f"{self.filename}: not an HDF5 file (no superblock signature)")
        ver = int(mm[base + 8])
        if ver in (0, 1):
            so, sl = int(mm[base + 13]), int(mm[base + 14])
            b = _Buf(mm, so, sl)
            p = base + 24 + (4 if ver == 1 else 0)
            self._base = b.off(p) if b.off(p) != UNDEF else base
            p += 4 * so                      # base, free space, EOF, driver info
            # root symbol table entry: link name offset, object header address
            self._root = b.off(p + so)
        elif ver in (2, 3):
            so, sl = int(mm[base + 9]), int(mm[base + 10])
            b = _Buf(mm, so, sl)
            p = base + 12
            self._base = b.off(p)
            self._root = b.off(p + 3 * so)
        else:
            raise H5Error(f"superblock version {ver} is not supported")
        self._b = b
        if self._base == UNDEF:
            self._base = base

    def close(self):
        self._mm = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- object headers -------------------------------------------------
    def _messages(self, addr):
        """(type, data offset, size) of every message of an object header."""
        b, a = self._b, self._base + addr
        out = []
        if bytes(b.mm[a:a + 4]) == b"OHDR":
            version = int(b.mm[a + 4])
            if version != 2:
                raise H5Error(f"object header version {version} at {addr} is not supported")
            flags = int(b.mm[a + 5])
            p = a + 6
            if flags & 0x20:
                p += 16                      # access/modify/change/birth times
            if flags & 0x10:
                p += 4                       # attribute phase change values
            nsz = 1 << (flags & 3)
            size0 = b.u(p, nsz)
            p += nsz
            blocks = [(p, size0)]
            crt = bool(flags & 0x04)
            while blocks:
                start, size = blocks.pop(0)
                q, end = start, start + size
                while q + 4 <= end:
                    mtype, msize = int(b.mm[q]), b.u(q + 1, 2)
                    q += 4 + (2 if crt else 0)
                    if mtype == 0x10:        # continuation: OCHK block
                        ca, cl = b.off(q), b.ln(q + b.so)
                        b.sig(self._base + ca, b"OCHK")
                        blocks.append((self._base + ca + 4, cl - 8))
                    elif mtype != 0:
                        out.append((mtype, q, msize))
                    q += msize
            return out
        version = int(b.mm[a])
        if version != 1:
            raise H5Error(f"object header at {addr}: version {version} is not supported")
        nmsg = b.u(a + 2, 2)
        hsize = b.u(a + 8, 4)
        blocks = [(a + 16, hsize)]
        while blocks and len(out) < nmsg + 64:
            start, size = blocks.pop(0)
            q, end = start, start + size
            while q + 8 <= end:
                mtype, msize = b.u(q, 2), b.u(q + 2, 2)
                q += 8
                if mtype == 0x10:
                    blocks.append((self._base + b.off(q), b.ln(q + b.so)))
                elif mtype != 0:
                    out.append((mtype, q, msize))
                q += msize
        return out

    # ---- groups ---------------------------------------------------------
    def _group_members(self, addr):
        """{name: object header address} of a group."""
        b = self._b
        members = {}
        for mtype, p, _ in self._messages(addr):
            if mtype == 0x11:                # symbol table: B-tree + local heap
                members.update(self._symbol_table(b.off(p), b.off(p + b.so)))
            elif mtype == 0x06:              # link message (compact group)
                name, target = self._link(p)
                if target is not None:
                    members[name] = target
            elif mtype == 0x02:              # link info: dense storage?
                flags = int(b.mm[p + 1])
                q = p + 2 + (8 if flags & 1 else 0)
                if b.off(q) != UNDEF:
                    raise H5Error("groups in dense (fractal heap) storage are not supported")
        return members

    def _link(self, p):
        b = self._b
        flags = int(b.mm[p + 1])
        q = p + 2
        ltype = 0
        if flags & 0x08:
            ltype = int(b.mm[q])
            q += 1
        if flags & 0x04:
            q += 8
        if flags & 0x10:
            q += 1
        nlen_size = 1 << (flags & 3)
        nlen = b.u(q, nlen_size)
        q += nlen_size
        name = bytes(b.mm[q:q + nlen]).decode("utf-8")
        q += nlen
        if ltype != 0:
            return name, None               # soft or external link: not followed
        return name, b.off(q)

    def _heap(self, addr):
        b, a = self._b, self._base + addr
        b.sig(a, b"HEAP")
        return self._base + b.off(a + 8 + 2 * b.sl)

    def _symbol_table(self, btree, heap):
        b = self._b
        data = self._heap(heap)
        members = {}

        def name_at(off):
            s = data + off
            e = s
            while b.mm[e] != 0:
                e += 1
            return bytes(b.mm[s:e]).decode("utf-8")

        def walk(node):
            a = self._base + node
            b.sig(a, b"TREE")
            if int(b.mm[a + 4]) != 0:
                raise H5Error("symbol-table B-tree of unexpected node type")
            level, used = int(b.mm[a + 5]), b.u(a + 6, 2)
            p = a + 8 + 2 * b.so + b.sl      # skip siblings and key 0
            for _ in range(used):
                child = b.off(p)
                if level > 0:
                    walk(child)
                else:
                    snod = self._base + child
                    b.sig(snod, b"SNOD")
                    n = b.u(snod + 6, 2)
                    e = snod + 8
                    for _ in range(n):
                        members[name_at(b.off(e))] = b.off(e + b.so)
                        e += 2 * b.so + 24
                p += b.so + b.sl

        walk(btree)
        return members

    def _resolve(self, path):
        addr = self._root
        for part in [x for x in path.split("/") if x]:
            members = self._group_members(addr)
            if part not in members:
                raise H5Error(f"{self.filename}: no object {path!r} (missing {part!r})")
            addr = members[part]
        return addr

    # ---- datasets -------------------------------------------------------
    def _dtype(self, p):
        b = self._b
        cv = int(b.mm[p])
        cls = cv & 0x0F
        bits0 = int(b.mm[p + 1])
        size = b.u(p + 4, 4)
        order = ">" if bits0 & 1 else "<"
        if cls == 1 and size in (2, 4, 8):
            return np.dtype(f"{order}f{size}")
        if cls == 0 and size in (1, 2, 4, 8):
            return np.dtype(f"{order}{'i' if bits0 & 0x08 else 'u'}{size}")
        raise H5Error(f"datatype class {cls} of size {size} is not supported")

    def _dataspace(self, p):
        b = self._b
        version, rank, flags = int(b.mm[p]), int(b.mm[p + 1]), int(b.mm[p + 2])
        if version == 1:
            q = p + 8
        elif version == 2:
            if int(b.mm[p + 3]) == 2:
                return ()                   # null dataspace
            q = p + 4
        else:
            raise H5Error(f"dataspace version {version} is not supported")
        return tuple(b.ln(q + i * b.sl) for i in range(rank))

    def _dataset(self, path):
        b = self._b
        addr = self._resolve(path)
        shape = dtype = None
        layout = None
        filters = False
        for mtype, p, msize in self._messages(addr):
            if mtype == 0x01:
                shape = self._dataspace(p)
            elif mtype == 0x03:
                dtype = self._dtype(p)
            elif mtype == 0x0B:
                nfilt = int(b.mm[p + 1])
                filters = nfilt > 0
            elif mtype == 0x08:
                layout = (p, msize)
        if shape is None or dtype is None or layout is None:
            raise H5Error(f"{path!r} is not a dataset")
        if filters:
            raise H5Error(f"{path!r} uses filters (compression); only unfiltered data is supported")
        p, _ = layout
        version, cls = int(b.mm[p]), int(b.mm[p + 1])
        if version not in (3, 4):
            raise H5Error(f"data layout version {version} is not supported")
        if cls == 0:                        # compact: raw data in the header
            size = b.u(p + 2, 2)
            return _Dataset(shape, dtype, "compact", p + 4 - self._base, size, None, None, None,
                            False)
        if cls == 1:
            return _Dataset(shape, dtype, "contiguous", b.off(p + 2), b.ln(p + 2 + b.so), None,
                            None, None, False)
        if cls != 2:
            raise H5Error(f"data layout class {cls} is not supported")
        if version == 3:
            rank1 = int(b.mm[p + 2])
            bt = b.off(p + 3)
            q = p + 3 + b.so
            dims = [b.u(q + 4 * i, 4) for i in range(rank1)]
            return _Dataset(shape, dtype, "chunked", None, None, tuple(dims[:-1]), "btree1", bt,
                            False)
        flags, rank1, enc = int(b.mm[p + 2]), int(b.mm[p + 3]), int(b.mm[p + 4])
        q = p + 5
        dims = [b.u(q + enc * i, enc) for i in range(rank1)]
        q += enc * rank1
        itype = int(b.mm[q])
        q += 1
        if itype == 1:                      # single chunk
            if flags & 0x02:
                q += b.sl + 4               # filtered size and mask
            return _Dataset(shape, dtype, "chunked", None, None, tuple(dims[:-1]), "single",
                            b.off(q), False)
        if itype == 2:                      # implicit: chunks in order, no index
            return _Dataset(shape, dtype, "chunked", None, None, tuple(dims[:-1]), "implicit",
                            b.off(q), False)
        raise H5Error(f"chunk index type {itype} (fixed/extensible array, v2 B-tree) "
                      "is not supported")

    def _chunks(self, ds):
        """(chunk offset tuple, file address) of every stored chunk."""
        b = self._b
        rank = len(ds.shape)
        if ds.index == "single":
            return [((0,) * rank, ds.index_addr)]
        if ds.index == "implicit":
            grid = [-(-n // c) for n, c in zip(ds.shape, ds.chunk)]
            nbytes = int(np.prod(ds.chunk)) * ds.dtype.itemsize
            out = []
            for i, idx in enumerate(np.ndindex(*grid)):
                out.append((tuple(k * c for k, c in zip(idx, ds.chunk)), ds.index_addr + i * nbytes))
            return out
        out = []
        ksize = 8 + 8 * (rank + 1)

        def walk(node):
            a = self._base + node
            b.sig(a, b"TREE")
            if int(b.mm[a + 4]) != 1:
                raise H5Error("chunk B-tree of unexpected node type")
            level, used = int(b.mm[a + 5]), b.u(a + 6, 2)
            p = a + 8 + 2 * b.so
            for _ in range(used):
                offs = tuple(b.u(p + 8 + 8 * i, 8) for i in range(rank))
                child = b.off(p + ksize)
                if level > 0:
                    walk(child)
                else:
                    out.append((offs, child))
                p += ksize + b.so

        walk(ds.index_addr)
        return out

    def _array(self, ds):
        """The whole dataset: a read-only memory map where the layout allows."""
        if ds.layout in ("contiguous", "compact"):
            if ds.addr == UNDEF:
                return np.zeros(ds.shape, ds.dtype)     # never written: fill value 0
            return np.ndarray(ds.shape, ds.dtype, buffer=self._mm,
                              offset=self._base + ds.addr)
        out = np.zeros(ds.shape, ds.dtype)
        for offs, addr in self._chunks(ds):
            chunk = np.ndarray(ds.chunk, ds.dtype, buffer=self._mm, offset=self._base + addr)
            sl_out = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, ds.chunk, ds.shape))
            sl_in = tuple(slice(0, x.stop - x.start) for x in sl_out)
            out[sl_out] = chunk[sl_in]
        return out

    # ---- the reference Reader's calls ------------------------------------
    def shape(self, dataset):
        return self._dataset(dataset).shape

    def dims(self, dataset, dim):
        """Extent of dimension ``dim`` of a 3-D dataset (``Reader::dims``)."""
        shp = self.shape(dataset)
        if len(shp) != 3:
            raise H5Error("Data is not 3D")
        if dim < 0 or dim > 2:
            raise H5Error("Invalid dimension")
        return int(shp[dim])

    def _as_float32(self, a, dataset, strict):
        if a.dtype == np.dtype("<f4"):
            return a
        if strict:
            raise H5Error(f"{dataset!r}: data type mismatch ({a.dtype}, float32 wanted)")
        return a.astype(np.float32)

    def psd(self, dataset, strict=True):
        """The ``[projections][slices][detector]`` float32 dataset as an array
        (a memory map for contiguous layouts), without reordering."""
        ds = self._dataset(dataset)
        if len(ds.shape) != 3:
            raise H5Error("Data is not 3D")
        return self._as_float32(self._array(ds), dataset, strict)

    def read_sinogram(self, dataset, begin=0, end=-1, strict=True):
        """Slices ``begin .. end-1`` of a ``[P][S][D]`` dataset as a host array
        ``[slices][P][D]`` (``Reader::read_sinogram``)."""
        a = self.psd(dataset, strict)
        P, S, D = a.shape
        end = S if end == -1 else end
        if begin < 0 or end > S or end < begin:
            raise H5Error("Index out of bounds")
        return np.ascontiguousarray(a[:, begin:end, :].transpose(1, 0, 2))

    def read2(self, dataset, begin=0, end=-1, strict=True):
        """Leading-dimension slab ``begin .. end-1`` of a 3-D dataset
        (``Reader::read2``)."""
        a = self.psd(dataset, strict)
        end = a.shape[0] if end == -1 else end
        if begin < 0 or end > a.shape[0] or end < begin:
            raise H5Error("Index out of bounds")
        return np.array(a[begin:end])

    def read(self, dataset, strict=False):
        """A 1-D dataset, e.g. the projection angles (``Reader::read``)."""
        ds = self._dataset(dataset)
        return np.array(self._as_float32(self._array(ds), dataset, strict)).reshape(-1)

    def sinogram_to_device(self, dataset, begin=0, end=-1, out=None):
        """Slices ``begin .. end-1`` straight into device memory as
        ``[slices][P][D]`` (``tc_sino_ingest_psd``: one strided copy per
        projection out of the mapped file, no host transpose)."""
        from .ingest import sinogram_from_psd
        a = self.psd(dataset)
        S = a.shape[1]
        end = S if end == -1 else end
        return sinogram_from_psd(a, begin, end - begin, out=out)


# ---------------------------------------------------------------------------
# writing (the layout libhdf5 writes by default: superblock 0, version-1
# object headers, symbol-table groups)
# ---------------------------------------------------------------------------
_GROUP_LEAF_K, _GROUP_NODE_K, _CHUNK_K = 4, 16, 32


def _pad8(n):
    return (n + 7) & ~7


def _msg(mtype, body):
    body = body + b"\0" * (_pad8(len(body)) - len(body))
    return struct.pack("<HHB3x", mtype, len(body), 0) + body


def _ohdr(messages):
    data = b"".join(messages)
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(data)) + data


def _dtype_msg(dt):
    dt = np.dtype(dt)
    order = 1 if dt.byteorder == ">" else 0
    if dt.kind == "f":
        if dt.itemsize == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        elif dt.itemsize == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        else:
            raise H5Error(f"cannot write {dt}")
        bits = bytes([0x20 | order, dt.itemsize * 8 - 1, 0])
        return struct.pack("<B", 0x11) + bits + struct.pack("<I", dt.itemsize) + props
    if dt.kind in "iu":
        bits = bytes([order | (0x08 if dt.kind == "i" else 0), 0, 0])
        return (struct.pack("<B", 0x10) + bits + struct.pack("<I", dt.itemsize) +
                struct.pack("<HH", 0, dt.itemsize * 8))
    raise H5Error(f"cannot write {dt}")


class Writer:
    """Write float / integer datasets into a new HDF5 file
    (``src/hdf5/writer.h`` ``Writer::write``).  Paths may name groups
    ("/exchange/data"); the file is written on close()."""

    def __init__(self, filename):
        self.filename = os.fspath(filename)
        self._tree = {}

    def write(self, name, array, chunks=None):
        parts = [x for x in name.split("/") if x]
        if not parts:
            raise H5Error("empty dataset name")
        node = self._tree
        for g in parts[:-1]:
            node = node.setdefault(g, {})
            if not isinstance(node, dict):
                raise H5Error(f"{g!r} is a dataset")
        a = np.asarray(array)
        if a.dtype.kind not in "fiu":
            raise H5Error(f"cannot write {a.dtype}")
        if chunks is not None:
            chunks = tuple(int(c) for c in chunks)
            if len(chunks) != a.ndim or min(chunks) < 1:
                raise H5Error("chunk shape must have one positive extent per dimension")
        node[parts[-1]] = (np.ascontiguousarray(a), chunks)

    def close(self):
        out = bytearray(96)                 # superblock, written last
        pos = [96]

        def alloc(n):
            a = pos[0]
            pos[0] += _pad8(n)
            out.extend(b"\0" * (pos[0] - len(out)))
            return a

        def put(addr, data):
            out[addr:addr + len(data)] = data

        def write_dataset(a, chunks):
            msgs_len = lambda body: 8 + _pad8(len(body))  # noqa: E731
            space = struct.pack("<BBBx4x", 1, a.ndim, 0) + b"".join(
                struct.pack("<Q", d) for d in a.shape)
            dtm = _dtype_msg(a.dtype)
            fill = struct.pack("<BBBB", 2, 3 if chunks else 2, 2, 0)
            if chunks is None:
                layout_len = 18
            else:
                layout_len = 3 + 8 + 4 * (a.ndim + 1)
            hlen = 16 + sum(msgs_len(x) for x in (space, dtm, fill)) + 8 + _pad8(layout_len)
            hdr = alloc(hlen)
            if chunks is None:
                data = alloc(a.nbytes)
                put(data, a.tobytes())       # in the byte order the datatype message states
                layout = struct.pack("<BBQQ", 3, 1, data, a.nbytes)
            else:
                grid = [-(-n // c) for n, c in zip(a.shape, chunks)]
                offsets = [tuple(i * c for i, c in zip(idx, chunks)) for idx in np.ndindex(*grid)]
                if len(offsets) > 2 * _CHUNK_K:
                    raise H5Error(f"at most {2 * _CHUNK_K} chunks per dataset")
                rank1 = a.ndim + 1
                ksize = 8 + 8 * rank1
                node_len = 8 + 16 + (2 * _CHUNK_K + 1) * ksize + 2 * _CHUNK_K * 8
                node = alloc(node_len)
                nbytes = int(np.prod(chunks)) * a.dtype.itemsize
                body = bytearray(struct.pack("<4sBBHQQ", b"TREE", 1, 0, len(offsets), UNDEF, UNDEF))
                for off in offsets:
                    c = np.zeros(chunks, a.dtype)
                    sl = tuple(slice(o, min(o + ch, n)) for o, ch, n in zip(off, chunks, a.shape))
                    c[tuple(slice(0, x.stop - x.start) for x in sl)] = a[sl]
                    caddr = alloc(nbytes)
                    put(caddr, c.tobytes())
                    body += struct.pack("<II", nbytes, 0) + b"".join(
                        struct.pack("<Q", o) for o in off) + struct.pack("<Q", 0)
                    body += struct.pack("<Q", caddr)
                body += struct.pack("<II", 0, 0) + b"".join(
                    struct.pack("<Q", n) for n in a.shape) + struct.pack("<Q", 0)
                put(node, bytes(body))
                layout = struct.pack("<BBBQ", 3, 2, rank1, node) + b"".join(
                    struct.pack("<I", c) for c in chunks) + struct.pack("<I", a.dtype.itemsize)
            put(hdr, _ohdr([_msg(0x01, space), _msg(0x03, dtm), _msg(0x05, fill),
                            _msg(0x08, layout)]))
            return hdr

        def write_group(tree):
            """Returns (object header, B-tree, local heap) addresses."""
            names = sorted(tree)
            if len(names) > 2 * _GROUP_LEAF_K * 2 * _GROUP_NODE_K:
                raise H5Error("too many members in one group")
            targets = {}
            for n in names:
                v = tree[n]
                if isinstance(v, dict):
                    targets[n] = (write_group(v), True)
                else:
                    targets[n] = ((write_dataset(*v), None, None), False)
            # local heap: "" at offset 0, then the names
            heapdata = bytearray(8)
            name_off = {}
            for n in names:
                name_off[n] = len(heapdata)
                enc = n.encode("utf-8") + b"\0"
                heapdata += enc + b"\0" * (_pad8(len(enc)) - len(enc))
            heap = alloc(32)
            seg = alloc(len(heapdata))
            put(seg, bytes(heapdata))
            # no free block: libhdf5 marks the empty free list with offset 1
            put(heap, struct.pack("<4sB3xQQQ", b"HEAP", 0, len(heapdata), 1, seg))
            # symbol nodes of 2 * leaf K entries
            cap = 2 * _GROUP_LEAF_K
            groups = [names[i:i + cap] for i in range(0, len(names), cap)] or [[]]
            snod_len = 8 + cap * 40
            snods = []
            for grp in groups:
                sn = alloc(snod_len)
                body = bytearray(struct.pack("<4sBBH", b"SNOD", 1, 0, len(grp)))
                for n in grp:
                    (oh, bt, hp), is_group = targets[n]
                    if is_group:
                        body += struct.pack("<QQI4xQQ", name_off[n], oh, 1, bt, hp)
                    else:
                        body += struct.pack("<QQI4x16x", name_off[n], oh, 0)
                put(sn, bytes(body))
                snods.append((sn, grp))
            node_len = 8 + 16 + (2 * _GROUP_NODE_K + 1) * 8 + 2 * _GROUP_NODE_K * 8
            bt = alloc(node_len)
            body = bytearray(struct.pack("<4sBBHQQ", b"TREE", 0, 0, len(snods) if names else 0,
                                         UNDEF, UNDEF))
            body += struct.pack("<Q", 0)
            if names:
                for sn, grp in snods:
                    body += struct.pack("<QQ", sn, name_off[grp[-1]])
            put(bt, bytes(body))
            oh = alloc(16 + 8 + 16)
            put(oh, _ohdr([_msg(0x11, struct.pack("<QQ", bt, heap))]))
            return oh, bt, heap

        root_oh, root_bt, root_heap = write_group(self._tree)
        eof = len(out)
        sb = struct.pack("<8sBBBBBBBBHHI", SIGNATURE, 0, 0, 0, 0, 0, 8, 8, 0, _GROUP_LEAF_K,
                         _GROUP_NODE_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQI4xQQ", 0, root_oh, 1, root_bt, root_heap)
        assert len(sb) == 96
        out[0:96] = sb
        with open(self.filename, "wb") as f:
            f.write(bytes(out))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if exc[0] is None:
            self.close()
