"""A small reader and writer of the HDF5 subset that redrock's details files
use (redrock 0.22 results.py: h5py writes them with its default settings).

The subset, from the published HDF5 file-format specification:
  * superblock version 0 (8-byte offsets and lengths);
  * version-1 object headers (with continuation blocks);
  * groups as symbol tables: a version-1 group B-tree, symbol-table nodes
    ("SNOD") and a local heap of link names;
  * datasets with a dataspace, a datatype, a fill-value message and a
    contiguous (or compact) version-3 layout, no filters;
  * datatypes: fixed-point, IEEE floating point, fixed-length strings,
    compounds (member versions 1-3) and arrays (versions 2-3).

Reading covers the files redrock writes through h5py; writing produces the
same structures (one-level group B-trees, whose fan-out is set in the
superblock to fit the largest group).  h5py is not needed for either.
"""

from __future__ import annotations

import os
import struct

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF
_HEAP_FREE_NULL = 1          # "no free block" in a local heap's free list


class HDF5FormatError(ValueError):
    pass


# ---------------------------------------------------------------------------
# reading
# ---------------------------------------------------------------------------

class _Reader:
    def __init__(self, data):
        self.d = data
        if data[:8] != _SIG:
            raise HDF5FormatError("not an HDF5 file")
        if data[8] != 0:
            raise HDF5FormatError(f"superblock version {data[8]} is not supported")
        if data[13] != 8 or data[14] != 8:
            raise HDF5FormatError("only 8-byte offsets and lengths are supported")
        # root group symbol table entry after the 4 addresses
        self.root = self.u64(24 + 32 + 8)

    def u16(self, o):
        return struct.unpack_from("<H", self.d, o)[0]

    def u32(self, o):
        return struct.unpack_from("<I", self.d, o)[0]

    def u64(self, o):
        return struct.unpack_from("<Q", self.d, o)[0]

    def messages(self, addr):
        d = self.d
        if d[addr] != 1:
            raise HDF5FormatError(f"object header version {d[addr]} is not supported")
        n = self.u16(addr + 2)
        blocks = [(addr + 16, self.u32(addr + 8))]
        out = []
        while blocks and len(out) < n:
            o, size = blocks.pop(0)
            end = o + size
            while o + 8 <= end and len(out) < n:
                t, s = self.u16(o), self.u16(o + 2)
                out.append((t, o + 8, s))
                if t == 0x10:
                    blocks.append((self.u64(o + 8), self.u64(o + 16)))
                o += 8 + s
        return out

    def heap_name(self, heap, off):
        if self.d[heap:heap + 4] != b"HEAP":
            raise HDF5FormatError("bad local heap")
        seg = self.u64(heap + 24)
        e = self.d.index(b"\0", seg + off)
        return self.d[seg + off:e].decode()

    def links(self, btree, heap):
        d = self.d
        if d[btree:btree + 4] != b"TREE":
            raise HDF5FormatError("bad group B-tree")
        level, n = d[btree + 5], self.u16(btree + 6)
        out = []
        o = btree + 24
        for _ in range(n):
            child = self.u64(o + 8)
            o += 16
            if level > 0:
                out += self.links(child, heap)
                continue
            if d[child:child + 4] != b"SNOD":
                raise HDF5FormatError("bad symbol table node")
            for k in range(self.u16(child + 6)):
                e = child + 8 + 40 * k
                out.append((self.heap_name(heap, self.u64(e)), self.u64(e + 8)))
        return out

    # -- datatypes ---------------------------------------------------------
    def dtype(self, o):
        """(numpy dtype, bytes used) of the datatype message at o."""
        d = self.d
        cls, ver = d[o] & 0x0F, d[o] >> 4
        bits = d[o + 1] | (d[o + 2] << 8) | (d[o + 3] << 16)
        size = self.u32(o + 4)
        p = o + 8
        if cls == 0:
            order = ">" if bits & 1 else "<"
            kind = "i" if bits & 8 else "u"
            return np.dtype(f"{order}{kind}{size}"), 12
        if cls == 1:
            order = ">" if bits & 1 else "<"
            return np.dtype(f"{order}f{size}"), 20
        if cls == 3:
            return np.dtype(f"S{size}"), 8
        if cls == 6:
            nmemb = bits & 0xFFFF
            names, formats, offsets = [], [], []
            for _ in range(nmemb):
                e = d.index(b"\0", p)
                name = d[p:e].decode()
                if ver < 3:
                    p += ((e - p) // 8 + 1) * 8
                    off = self.u32(p)
                    p += 4
                else:
                    p = e + 1
                    nb = 1 if size < 256 else 2 if size < 65536 else 3 if size < (1 << 24) else 4
                    off = int.from_bytes(d[p:p + nb], "little")
                    p += nb
                shape = ()
                if ver == 1:
                    rank = d[p]
                    dims = [self.u32(p + 12 + 4 * k) for k in range(rank)]
                    shape = tuple(dims)
                    p += 28
                mt, used = self.dtype(p)
                p += used
                names.append(name)
                formats.append((mt, shape) if shape else mt)
                offsets.append(off)
            return np.dtype({"names": names, "formats": formats, "offsets": offsets,
                             "itemsize": size}), p - o
        if cls == 10:
            rank = d[p]
            if ver == 2:
                dims = [self.u32(p + 4 + 4 * k) for k in range(rank)]
                q = p + 4 + 8 * rank
            else:
                dims = [self.u32(p + 1 + 4 * k) for k in range(rank)]
                q = p + 1 + 4 * rank
            base, used = self.dtype(q)
            return np.dtype((base, tuple(dims))), q + used - o
        raise HDF5FormatError(f"datatype class {cls} is not supported")

    def dataset(self, addr):
        shape = dt = raw = None
        for t, o, s in self.messages(addr):
            d = self.d
            if t == 0x01:
                ver, rank = d[o], d[o + 1]
                base = o + (8 if ver == 1 else 4)
                shape = tuple(self.u64(base + 8 * k) for k in range(rank))
            elif t == 0x03:
                dt, _ = self.dtype(o)
            elif t == 0x0B:
                raise HDF5FormatError("filtered (compressed) datasets are not supported")
            elif t == 0x08:
                if d[o] != 3:
                    raise HDF5FormatError(f"layout version {d[o]} is not supported")
                if d[o + 1] == 1:
                    raw = (self.u64(o + 2), self.u64(o + 10))
                elif d[o + 1] == 0:
                    raw = (o + 4, self.u16(o + 2))
                else:
                    raise HDF5FormatError("chunked datasets are not supported")
        if shape is None or dt is None or raw is None:
            raise HDF5FormatError("incomplete dataset header")
        n = int(np.prod(shape)) if shape else 1
        if raw[0] == _UNDEF:
            return np.zeros(shape, dtype=dt)
        a = np.frombuffer(self.d, dtype=dt, count=n, offset=raw[0]).reshape(shape)
        return a.copy()


class Group:
    """A group of an HDF5 file opened with ``File``: ``keys()`` in name
    order, ``g[name]`` a Group or a numpy array, paths with '/'."""

    def __init__(self, reader, addr):
        self._r = reader
        self._addr = addr
        self._links = None

    def _table(self):
        if self._links is None:
            stab = [o for t, o, s in self._r.messages(self._addr) if t == 0x11]
            if not stab:
                raise HDF5FormatError("not a group")
            bt, heap = self._r.u64(stab[0]), self._r.u64(stab[0] + 8)
            self._links = dict(self._r.links(bt, heap))
        return self._links

    def keys(self):
        return list(self._table().keys())

    def __contains__(self, name):
        try:
            self[name]
            return True
        except KeyError:
            return False

    def __getitem__(self, path):
        node = self
        for part in [p for p in path.split("/") if p]:
            if not isinstance(node, Group):
                raise KeyError(path)
            addr = node._table().get(part)
            if addr is None:
                raise KeyError(path)
            if any(t == 0x11 for t, _, _ in node._r.messages(addr)):
                node = Group(node._r, addr)
            else:
                node = node._r.dataset(addr)
        return node


class File(Group):
    """Read-only HDF5 file (the whole file is read into memory)."""

    def __init__(self, filename, mode="r"):
        if mode != "r":
            raise ValueError("use write_file to write")
        with open(os.path.expandvars(filename), "rb") as f:
            data = f.read()
        r = _Reader(data)
        super().__init__(r, r.root)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def close(self):
        pass


# ---------------------------------------------------------------------------
# writing
# ---------------------------------------------------------------------------

def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def _dtype_msg(dt):
    """Datatype message body for a numpy dtype."""
    dt = np.dtype(dt)
    if dt.subdtype is not None:
        base, shape = dt.subdtype
        body = bytes([len(shape), 0, 0, 0]) + b"".join(struct.pack("<I", s) for s in shape)
        body += b"".join(struct.pack("<I", k) for k in range(len(shape)))
        return (struct.pack("<B3sI", 0x2A, b"\0\0\0", dt.itemsize) + body + _dtype_msg(base))
    if dt.names:
        body = b""
        for name in dt.names:
            ft, off = dt.fields[name][:2]
            body += _pad8(name.encode() + b"\0") + struct.pack("<I", off) + _dtype_msg(ft)
        n = len(dt.names)
        return struct.pack("<B", 0x26) + bytes([n & 0xFF, n >> 8, 0]) + \
            struct.pack("<I", dt.itemsize) + body
    order = 1 if dt.byteorder == ">" else 0
    if dt.kind in "iu":
        bits = order | (8 if dt.kind == "i" else 0)
        return struct.pack("<B3sI", 0x10, bytes([bits, 0, 0]), dt.itemsize) + \
            struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "f":
        if dt.itemsize == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
            bits = order | 0x20 | (0x3F << 8)  # IEEE, msb-set mantissa norm, sign bit 63
        elif dt.itemsize == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
            bits = order | 0x20 | (0x1F << 8)
        else:
            raise HDF5FormatError(f"float of {dt.itemsize} bytes is not supported")
        return struct.pack("<B3sI", 0x11, bytes([bits & 0xFF, bits >> 8, 0]), dt.itemsize) + props
    if dt.kind == "S":
        return struct.pack("<B3sI", 0x13, bytes([1, 0, 0]), dt.itemsize)
    raise HDF5FormatError(f"numpy dtype {dt} is not supported")


class _Writer:
    def __init__(self):
        self.buf = bytearray()

    def alloc(self, n):
        o = len(self.buf)
        self.buf += b"\0" * (n + (-n % 8))
        return o

    def put(self, o, b):
        self.buf[o:o + len(b)] = b

    def object_header(self, msgs):
        """msgs: [(type, body, flags)] -> address of a v1 object header."""
        body = b""
        for t, b, fl in msgs:
            b = _pad8(b)
            body += struct.pack("<HHB3s", t, len(b), fl, b"\0\0\0") + b
        o = self.alloc(16 + len(body))
        self.put(o, struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + b"\0" * 4 + body)
        return o

    def dataset(self, arr):
        arr = np.ascontiguousarray(arr)
        if arr.dtype.byteorder == ">" or (arr.dtype.names and any(
                arr.dtype.fields[n][0].byteorder == ">" for n in arr.dtype.names)):
            raise HDF5FormatError("big-endian arrays are not supported")
        data = arr.tobytes()
        daddr = self.alloc(len(data)) if data else _UNDEF
        if data:
            self.put(daddr, data)
        shape = arr.shape
        space = struct.pack("<BBBB4s", 1, len(shape), 1, 0, b"\0" * 4)
        space += b"".join(struct.pack("<Q", s) for s in shape) * 2
        fill = bytes([2, 2, 2, 1, 0, 0, 0, 0])
        layout = struct.pack("<BBQQ", 3, 1, daddr, len(data))
        return self.object_header([(0x01, space, 0), (0x03, _dtype_msg(arr.dtype), 1),
                                   (0x05, fill, 1), (0x08, layout, 0)])

    def group(self, entries, leaf_k, node_k):
        """entries: {name: (addr, stab or None)} -> (header addr, btree, heap)."""
        names = sorted(entries, key=lambda s: s.encode())
        seg = b"\0" * 8
        offs = {}
        for n in names:
            offs[n] = len(seg)
            seg += _pad8(n.encode() + b"\0")
        heap = self.alloc(32)
        segaddr = self.alloc(len(seg))
        self.put(segaddr, seg)
        self.put(heap, b"HEAP" + struct.pack("<B3sQQQ", 0, b"\0\0\0", len(seg), _HEAP_FREE_NULL,
                                             segaddr))
        per = 2 * leaf_k
        chunks = [names[i:i + per] for i in range(0, len(names), per)] or [[]]
        if len(chunks) > 2 * node_k:
            raise HDF5FormatError("group too large for the B-tree fan-out")
        snods = []
        for ch in chunks:
            o = self.alloc(8 + 40 * per)
            body = b"SNOD" + struct.pack("<BBH", 1, 0, len(ch))
            for n in ch:
                addr, stab = entries[n]
                scratch = struct.pack("<QQ", *stab) if stab else b"\0" * 16
                body += struct.pack("<QQI4s", offs[n], addr, 1 if stab else 0, b"\0" * 4) + scratch
            self.put(o, body)
            snods.append(o)
        bt = self.alloc(24 + (2 * node_k + 1) * 8 + 2 * node_k * 8)
        body = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(snods) if names else 0, _UNDEF, _UNDEF)
        body += struct.pack("<Q", 0)
        if names:
            for o, ch in zip(snods, chunks):
                body += struct.pack("<QQ", o, offs[ch[-1]])
        self.put(bt, body)
        hdr = self.object_header([(0x11, struct.pack("<QQ", bt, heap), 0)])
        return hdr, bt, heap


def write_file(filename, tree):
    """Write a nested dict {name: dict (a group) or numpy array (a dataset)}
    as an HDF5 file (superblock 0, symbol-table groups, contiguous data)."""

    def count(node):
        n = len(node)
        return max([n] + [count(v) for v in node.values() if isinstance(v, dict)])

    leaf_k = 4
    node_k = max(16, -(-count(tree) // (2 * leaf_k) // 2) + 1)
    w = _Writer()
    w.alloc(96)  # superblock v0 with the root entry

    def build(node):
        entries = {}
        for name, v in node.items():
            if "/" in name:
                raise ValueError(f"'/' in name {name!r}")
            if isinstance(v, dict):
                hdr, bt, heap = build(v)
                entries[name] = (hdr, (bt, heap))
            else:
                entries[name] = (w.dataset(np.asarray(v)), None)
        return w.group(entries, leaf_k, node_k)

    hdr, bt, heap = build(tree)
    sb = _SIG + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, leaf_k, node_k, 0)
    sb += struct.pack("<QQQQ", 0, _UNDEF, len(w.buf), _UNDEF)
    sb += struct.pack("<QQI4sQQ", 0, hdr, 1, b"\0" * 4, bt, heap)
    w.put(0, sb)
    tmp = filename + ".tmp"
    with open(tmp, "wb") as f:
        f.write(bytes(w.buf))
    os.replace(tmp, filename)
