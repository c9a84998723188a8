"""A small HDF5 writer for tests of rrtmgp_b200.netcdf.

It writes the file-format structures that the reader decodes, in two styles: superblock
version 0 with version-1 object headers and groups as symbol tables (v1 B-tree of group nodes
+ local heap + symbol-table nodes), or superblock version 2 with version-2 object headers and
groups as link messages.  Datasets carry a version-1 dataspace, a fixed-point / floating-point /
fixed-length string datatype, and data layout version 3 (compact, contiguous, chunked with a
v1 B-tree chunk index of one or two levels) behind a filter pipeline of version 1 or 2
(shuffle, deflate, fletcher32).  The structures follow the HDF5 file-format specification;
checksums are written as zeros (the reader does not verify them).
"""
import itertools
import struct
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"
SHUFFLE, DEFLATE, FLETCHER32 = 2, 1, 3


class Dataset:
    """data: numpy array; layout: "contiguous" | "compact" | "chunked" | "unallocated";
    chunks: chunk shape; filters: list of filter ids applied in order; pipeline_version: 1 | 2;
    skip: {chunk index (tuple of offsets): filter mask} to store some chunks with filters skipped;
    leaf: chunks per B-tree leaf (a second level is written when there are several leaves)."""

    def __init__(self, data, layout="contiguous", chunks=None, filters=(), pipeline_version=1, skip=None, leaf=None):
        self.data = np.asarray(data)
        self.layout = layout
        self.chunks = chunks
        self.filters = list(filters)
        self.pipeline_version = pipeline_version
        self.skip = skip or {}
        self.leaf = leaf


class H5Writer:
    """version 0: superblock 0, version-1 object headers, groups as symbol tables;
    version 2: superblock 2, version-2 object headers ("OHDR"), groups as link messages (a link
    info message with no dense storage plus one hard-link message per member)."""

    def __init__(self, version=0):
        assert version in (0, 2)
        self.version = version
        self.b = bytearray(96 if version == 0 else 48)

    def _alloc(self, data):
        while len(self.b) % 8:
            self.b.append(0)
        addr = len(self.b)
        self.b += data
        return addr

    def _header(self, msgs):
        if self.version == 2:
            body = bytearray()
            for mtype, d in msgs:
                body += struct.pack("<BHB", mtype, len(d), 0) + d
            wide = len(body) > 255                            # flags bits 0-1: chunk-size width 1 or 2 bytes
            head = b"OHDR" + bytes([2, 0x01 if wide else 0x00])
            head += struct.pack("<H" if wide else "<B", len(body))
            return self._alloc(head + body + bytes(4))       # checksum (not verified by the reader)
        body = bytearray()
        for mtype, d in msgs:
            pad = (-len(d)) % 8
            body += struct.pack("<HHB3x", mtype, len(d) + pad, 0) + d + bytes(pad)
        return self._alloc(struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body)

    @staticmethod
    def _dataspace(shape):
        return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", n) for n in shape)

    @staticmethod
    def _datatype(dt):
        if dt.kind == "S":
            return bytes([0x13, 0x00, 0, 0]) + struct.pack("<I", dt.itemsize)
        order = 1 if dt.byteorder == ">" else 0
        if dt.kind in "iu":
            bits = order | (8 if dt.kind == "i" else 0)
            return bytes([0x10, bits, 0, 0]) + struct.pack("<IHH", dt.itemsize, 0, 8 * dt.itemsize)
        if dt.kind == "f":
            sign, eloc, esize, msize, bias = (63, 52, 11, 52, 1023) if dt.itemsize == 8 else (31, 23, 8, 23, 127)
            return (bytes([0x11, order | 0x20, sign, 0]) + struct.pack("<IHH", dt.itemsize, 0, 8 * dt.itemsize) +
                    bytes([eloc, esize, 0, msize]) + struct.pack("<I", bias))
        raise ValueError(dt)

    @staticmethod
    def _pipeline(ds):
        vals = {SHUFFLE: [ds.data.dtype.itemsize], DEFLATE: [6], FLETCHER32: []}
        if ds.pipeline_version == 1:
            out = struct.pack("<BB2x4x", 1, len(ds.filters))
            for fid in ds.filters:
                v = vals[fid]
                out += struct.pack("<HHHH", fid, 0, 0, len(v)) + b"".join(struct.pack("<I", x) for x in v)
                out += bytes(4) if len(v) % 2 else b""
            return out
        out = struct.pack("<BB", 2, len(ds.filters))
        for fid in ds.filters:
            v = vals[fid]
            out += struct.pack("<HHH", fid, 0, len(v)) + b"".join(struct.pack("<I", x) for x in v)
        return out

    @staticmethod
    def _apply(raw, filters, mask, itemsize):
        for i, fid in enumerate(filters):
            if mask & (1 << i):
                continue
            if fid == SHUFFLE:
                n = len(raw) // itemsize
                raw = np.frombuffer(raw, np.uint8).reshape(n, itemsize).T.tobytes()
            elif fid == DEFLATE:
                raw = zlib.compress(raw, 6)
            elif fid == FLETCHER32:
                raw = raw + bytes(4)
        return raw

    def _chunk_index(self, ds):
        a, cs = ds.data, tuple(ds.chunks)
        rank = a.ndim
        entries = []
        for idx in itertools.product(*[range(0, s, c) for s, c in zip(a.shape, cs)]):
            chunk = np.zeros(cs, a.dtype)
            src = tuple(slice(o, min(o + c, s)) for o, c, s in zip(idx, cs, a.shape))
            chunk[tuple(slice(0, x.stop - x.start) for x in src)] = a[src]
            mask = ds.skip.get(idx, 0)
            raw = self._apply(chunk.tobytes(), ds.filters, mask, a.dtype.itemsize)
            entries.append((len(raw), mask, idx, self._alloc(raw)))

        def key(size, mask, offs):
            return struct.pack("<II", size, mask) + b"".join(struct.pack("<Q", o) for o in offs) + struct.pack("<Q", 0)

        end_key = key(0, 0, a.shape)

        def node(level, items):
            # items: (key bytes, child address); the node holds key0 child0 ... keyN
            out = b"TREE" + bytes([1, level]) + struct.pack("<HQQ", len(items), UNDEF, UNDEF)
            for k, child in items:
                out += k + struct.pack("<Q", child)
            return self._alloc(out + end_key)

        leaf = ds.leaf or len(entries)
        groups = [entries[i:i + leaf] for i in range(0, len(entries), leaf)]
        leaves = [(key(g[0][0], g[0][1], g[0][2]), node(0, [(key(s, m, o), ad) for s, m, o, ad in g])) for g in groups]
        if len(leaves) == 1:
            return leaves[0][1]
        return node(1, leaves)

    def dataset(self, ds):
        a = ds.data
        msgs = [(0x01, self._dataspace(a.shape)), (0x03, self._datatype(a.dtype))]
        if ds.filters:
            msgs.append((0x0B, self._pipeline(ds)))
        if ds.layout == "compact":
            raw = a.tobytes()
            layout = bytes([3, 0]) + struct.pack("<H", len(raw)) + raw
        elif ds.layout == "contiguous":
            layout = bytes([3, 1]) + struct.pack("<QQ", self._alloc(a.tobytes()), a.nbytes)
        elif ds.layout == "unallocated":
            layout = bytes([3, 1]) + struct.pack("<QQ", UNDEF, a.nbytes)
        else:
            bt = self._chunk_index(ds)
            layout = (bytes([3, 2, a.ndim + 1]) + struct.pack("<Q", bt) +
                      b"".join(struct.pack("<I", c) for c in ds.chunks) + struct.pack("<I", a.dtype.itemsize))
        msgs.append((0x08, layout))
        return self._header(msgs)

    def group(self, members):
        """members: name -> Dataset or dict (a subgroup); returns the group's header address."""
        addrs = {}
        for name in sorted(members):
            m = members[name]
            addrs[name] = self.group(m) if isinstance(m, dict) else self.dataset(m)
        if self.version == 2:
            msgs = [(0x02, bytes([0, 0]) + struct.pack("<QQ", UNDEF, UNDEF))]    # link info, no dense links
            for name, addr in addrs.items():
                raw = name.encode()
                msgs.append((0x06, bytes([1, 0x08]) + bytes([0]) + bytes([len(raw)]) + raw + struct.pack("<Q", addr)))
            return self._header(msgs)
        heap = bytearray(8)                         # offset 0: the empty name
        offs = {}
        for name in sorted(addrs):
            offs[name] = len(heap)
            heap += name.encode() + b"\0"
            heap += bytes((-len(heap)) % 8)
        data = self._alloc(bytes(heap))
        lheap = self._alloc(b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap), UNDEF, data))
        snod = b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(addrs))
        for name in sorted(addrs):
            snod += struct.pack("<QQII", offs[name], addrs[name], 0, 0) + bytes(16)
        snod_addr = self._alloc(snod)
        last = offs[sorted(addrs)[-1]] if addrs else 0
        tree = (b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", 1, UNDEF, UNDEF) + struct.pack("<Q", 0) +
                struct.pack("<Q", snod_addr) + struct.pack("<Q", last))
        btree = self._alloc(tree)
        return self._header([(0x11, struct.pack("<QQ", btree, lheap))])

    def write(self, path, members):
        root = self.group(members)
        if self.version == 2:
            sb = SIG + bytes([2, 8, 8, 0]) + struct.pack("<QQQQ", 0, UNDEF, len(self.b), root) + bytes(4)
            assert len(sb) == 48
            self.b[:48] = sb
            with open(path, "wb") as f:
                f.write(bytes(self.b))
            return
        sb = (SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0) +
              struct.pack("<QQQQ", 0, UNDEF, len(self.b), UNDEF) + struct.pack("<QQII", 0, root, 0, 0) + bytes(16))
        assert len(sb) == 96
        self.b[:96] = sb
        with open(path, "wb") as f:
            f.write(bytes(self.b))
