"""A minimal reader and writer of the HDF5 file format for the FK-spectra file.

The image has no HDF5 library, so the structures the FK-spectra file needs are
written and read here from the published HDF5 file-format specification
(format version 0 objects, which the HDF5 library writes by default):

* superblock version 0 (8-byte offsets and lengths), found at byte 0 or
  after a user block of 512, 1024, ... bytes;
* version-1 object headers, with continuation messages;
* groups as symbol tables: a version-1 group B-tree over symbol-table nodes
  (SNOD), link names in a local heap;
* datasets with contiguous (or, on read, compact) layout;
* datatypes: little-endian signed 32-bit integers and IEEE floats, fixed-
  length ASCII strings; dataspaces: scalar and simple;
* attributes (version-1 attribute messages).

Anything else (superblock versions 2 and 3, version-2 object headers, chunked
or compressed datasets, dense attribute storage, variable-length types) is
rejected with H5FormatError, not guessed at.
"""
from __future__ import annotations

import os
import struct
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
HEAP_FREE_NULL = 1          # end of a local heap's free list
LEAF_K = 16                 # symbol-table node capacity 2K = 32 entries
INTERNAL_K = 16             # group B-tree node capacity 2K = 32 children
ENTRY_SIZE = 40             # symbol-table entry with 8-byte offsets and lengths
SNOD_SIZE = 8 + 2 * LEAF_K * ENTRY_SIZE
TREE_SIZE = 24 + (2 * INTERNAL_K + 1) * 8 + 2 * INTERNAL_K * 8

# header message types
MSG_NIL, MSG_DATASPACE, MSG_DATATYPE, MSG_FILL_OLD, MSG_FILL = 0x0, 0x1, 0x3, 0x4, 0x5
MSG_LAYOUT, MSG_ATTRIBUTE, MSG_CONTINUATION, MSG_STAB = 0x8, 0xC, 0x10, 0x11


class H5FormatError(ValueError):
    pass


def _pad8(n: int) -> int:
    return (n + 7) & ~7


# ---------------------------------------------------------------------------
#  Datatypes and dataspaces
# ---------------------------------------------------------------------------
def encode_datatype(dt) -> bytes:
    """Datatype message (version 1) of a numpy dtype: '<i4', '<f4', '<f8' or 'S<n>'."""
    dt = np.dtype(dt)
    if dt.kind == "i" and dt.byteorder in "<=":
        return struct.pack("<B3sIHH", 0x10, bytes([0x08, 0, 0]), dt.itemsize, 0, 8 * dt.itemsize)
    if dt.kind == "f" and dt.byteorder in "<=":
        if dt.itemsize == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
            bits = bytes([0x20, 31, 0])
        elif dt.itemsize == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
            bits = bytes([0x20, 63, 0])
        else:
            raise H5FormatError("unsupported float size %d" % dt.itemsize)
        return struct.pack("<B3sI", 0x11, bits, dt.itemsize) + props
    if dt.kind == "S":
        return struct.pack("<B3sI", 0x13, bytes([0x00, 0, 0]), dt.itemsize)   # null-terminated ASCII
    raise H5FormatError("unsupported datatype %s" % dt)


def decode_datatype(b: bytes) -> np.dtype:
    cls, ver = b[0] & 0x0F, b[0] >> 4
    bits = b[1:4]
    size = struct.unpack_from("<I", b, 4)[0]
    if ver not in (1, 2, 3):
        raise H5FormatError("datatype message version %d" % ver)
    if cls == 0:   # fixed point
        order = ">" if bits[0] & 1 else "<"
        return np.dtype("%s%s%d" % (order, "i" if bits[0] & 0x08 else "u", size))
    if cls == 1:   # floating point
        order = ">" if bits[0] & 1 else "<"
        if size not in (2, 4, 8):
            raise H5FormatError("float of %d bytes" % size)
        return np.dtype("%sf%d" % (order, size))
    if cls == 3:   # fixed-length string
        return np.dtype("S%d" % size)
    raise H5FormatError("datatype class %d is not supported" % cls)


def encode_dataspace(shape: Sequence[int]) -> bytes:
    """Dataspace message (version 1); shape () is scalar."""
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", int(d)) for d in shape)


def decode_dataspace(b: bytes) -> Tuple[int, ...]:
    ver, rank, flags = b[0], b[1], b[2]
    if ver == 1:
        off = 8
    elif ver == 2:
        if b[3] == 2:
            return (0,)   # null dataspace: no elements
        off = 4
    else:
        raise H5FormatError("dataspace message version %d" % ver)
    return tuple(struct.unpack_from("<%dQ" % rank, b, off)) if rank else ()


# ---------------------------------------------------------------------------
#  Writer
# ---------------------------------------------------------------------------
class _Dataset:
    def __init__(self, shape, dtype, data):
        self.shape, self.dtype, self.data = tuple(int(d) for d in shape), np.dtype(dtype), data
        self.attrs: Dict[str, np.ndarray] = {}
        self.addr = self.data_addr = 0
        self.nbytes = int(np.prod(self.shape, dtype=np.int64)) * self.dtype.itemsize


class _Group:
    def __init__(self):
        self.children: Dict[str, object] = {}
        self.attrs: Dict[str, np.ndarray] = {}
        self.addr = self.heap_addr = self.tree_addr = 0
        self.snod_addrs: List[int] = []


def _attr_value(value) -> np.ndarray:
    if isinstance(value, (str, bytes)):
        b = value.encode("ascii") if isinstance(value, str) else value
        return np.array(b, dtype="S%d" % max(1, len(b)))
    return np.ascontiguousarray(value)


def _attribute_message(name: str, value: np.ndarray) -> bytes:
    nb = name.encode("ascii") + b"\0"
    dt = encode_datatype(value.dtype)
    ds = encode_dataspace(value.shape)
    body = struct.pack("<BBHHH", 1, 0, len(nb), len(dt), len(ds))
    body += nb.ljust(_pad8(len(nb)), b"\0") + dt.ljust(_pad8(len(dt)), b"\0") + ds.ljust(_pad8(len(ds)), b"\0")
    return body + value.tobytes()


def _message(mtype: int, body: bytes, flags: int = 0) -> bytes:
    body = body.ljust(_pad8(len(body)), b"\0")
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _object_header(messages: List[bytes]) -> bytes:
    data = b"".join(messages)
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(data)) + data


class H5Writer:
    """Builds a file of groups, datasets and attributes, then lays it out.

    Datasets created with data=None are allocated but left to be filled later
    with write_rows / write_at (the file is sized, the region reads as zeros
    until written).  Usage: create_* and set_attr, then close() writes the
    metadata and the given data; deferred data may be written before or
    after close through the returned offsets."""

    def __init__(self, path: str):
        self.path = path
        self.root = _Group()
        self._laid_out = False

    def _parent(self, path: str) -> Tuple[_Group, str]:
        parts = [p for p in path.strip("/").split("/") if p]
        g = self.root
        for p in parts[:-1]:
            g = g.children[p]
            if not isinstance(g, _Group):
                raise H5FormatError("%s is not a group" % p)
        return g, parts[-1]

    def create_group(self, path: str) -> None:
        g, name = self._parent(path)
        g.children[name] = _Group()

    def create_dataset(self, path: str, data=None, shape=None, dtype=None) -> None:
        g, name = self._parent(path)
        if data is not None:
            data = np.ascontiguousarray(data)
            shape, dtype = data.shape, data.dtype
        g.children[name] = _Dataset(shape, dtype, data)

    def create_string(self, path: str, value: str) -> None:
        """Scalar fixed-length string dataset, as the reference's writeStringHDFWrapper makes it."""
        self.create_dataset(path, data=_attr_value(value))

    def set_attr(self, path: str, name: str, value) -> None:
        obj = self.root if path.strip("/") == "" else self._lookup(path)
        obj.attrs[name] = _attr_value(value)

    def _lookup(self, path: str):
        obj = self.root
        for p in [p for p in path.strip("/").split("/") if p]:
            obj = obj.children[p]
        return obj

    # ---- layout
    def _group_messages(self, g: _Group) -> List[bytes]:
        msgs = [_message(MSG_STAB, struct.pack("<QQ", g.tree_addr, g.heap_addr))]
        msgs += [_message(MSG_ATTRIBUTE, _attribute_message(n, v)) for n, v in g.attrs.items()]
        return msgs

    def _dataset_messages(self, d: _Dataset) -> List[bytes]:
        msgs = [_message(MSG_DATASPACE, encode_dataspace(d.shape)),
                _message(MSG_DATATYPE, encode_datatype(d.dtype), flags=1),   # constant
                _message(MSG_FILL, struct.pack("<BBBB", 2, 2, 2, 0)),
                _message(MSG_LAYOUT, struct.pack("<BBQQ", 3, 1, d.data_addr, d.nbytes))]
        msgs += [_message(MSG_ATTRIBUTE, _attribute_message(n, v)) for n, v in d.attrs.items()]
        return msgs

    @staticmethod
    def _heap(names: List[str]) -> Tuple[bytes, Dict[str, int]]:
        seg, offs = bytearray(8), {}   # offset 0: the empty name
        for n in names:
            offs[n] = len(seg)
            b = n.encode("ascii") + b"\0"
            seg += b.ljust(_pad8(len(b)), b"\0")
        return bytes(seg), offs

    def close(self) -> None:
        if self._laid_out:
            return
        # pass 1: addresses of every structure (metadata first, then the data regions)
        cursor = [96]   # after the superblock

        def alloc(n):
            a = cursor[0]
            cursor[0] += _pad8(n)
            return a

        objects = []

        def visit(g: _Group):
            names = sorted(g.children, key=lambda s: s.encode("ascii"))
            if len(names) > 2 * LEAF_K * 2 * INTERNAL_K:
                raise H5FormatError("group of %d members exceeds one B-tree level" % len(names))
            seg, offs = self._heap(names)
            g._names, g._offs, g._seg = names, offs, seg
            g.heap_addr = alloc(32)
            g._seg_addr = alloc(len(seg))
            g.tree_addr = alloc(TREE_SIZE)
            g.snod_addrs = [alloc(SNOD_SIZE) for _ in range(max(1, (len(names) + 2 * LEAF_K - 1) // (2 * LEAF_K)))]
            g.addr = alloc(len(_object_header(self._group_messages(g))))
            objects.append(g)
            for n in names:
                c = g.children[n]
                if isinstance(c, _Group):
                    visit(c)
                else:
                    c.addr = alloc(len(_object_header(self._dataset_messages(c))))
                    objects.append(c)

        visit(self.root)
        for o in objects:
            if isinstance(o, _Dataset):
                o.data_addr = alloc(o.nbytes) if o.nbytes else UNDEF
        eof = cursor[0]
        # pass 2: bytes
        with open(self.path, "wb") as fh:
            fh.truncate(eof)
            fh.seek(0)
            fh.write(SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, LEAF_K, INTERNAL_K, 0))
            fh.write(struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF))
            fh.write(struct.pack("<QQII", 0, self.root.addr, 1, 0) + struct.pack("<QQ", self.root.tree_addr,
                                                                               self.root.heap_addr))
            for o in objects:
                if isinstance(o, _Group):
                    self._write_group(fh, o)
                else:
                    fh.seek(o.addr)
                    fh.write(_object_header(self._dataset_messages(o)))
                    if o.data is not None and o.nbytes:
                        fh.seek(o.data_addr)
                        fh.write(np.ascontiguousarray(o.data, o.dtype).tobytes())
        self._laid_out = True

    def _write_group(self, fh, g: _Group) -> None:
        fh.seek(g.heap_addr)
        fh.write(b"HEAP" + struct.pack("<B3xQQQ", 0, len(g._seg), HEAP_FREE_NULL, g._seg_addr))
        fh.seek(g._seg_addr)
        fh.write(g._seg)
        chunks = [g._names[i:i + 2 * LEAF_K] for i in range(0, max(1, len(g._names)), 2 * LEAF_K)] or [[]]
        for addr, names in zip(g.snod_addrs, chunks):
            body = b"SNOD" + struct.pack("<BBH", 1, 0, len(names))
            for n in names:
                c = g.children[n]
                if isinstance(c, _Group):
                    body += struct.pack("<QQII", g._offs[n], c.addr, 1, 0) + struct.pack("<QQ", c.tree_addr, c.heap_addr)
                else:
                    body += struct.pack("<QQII", g._offs[n], c.addr, 0, 0) + bytes(16)
            fh.seek(addr)
            fh.write(body.ljust(SNOD_SIZE, b"\0"))
        # one leaf-level B-tree node over the symbol-table nodes: key 0 is the empty
        # name, key i+1 the last name of child i
        nchild = len(g.snod_addrs)
        tree = b"TREE" + struct.pack("<BBHQQ", 0, 0, nchild, UNDEF, UNDEF) + struct.pack("<Q", 0)
        for addr, names in zip(g.snod_addrs, chunks):
            tree += struct.pack("<QQ", addr, g._offs[names[-1]] if names else 0)
        fh.seek(g.tree_addr)
        fh.write(tree.ljust(TREE_SIZE, b"\0"))
        fh.seek(g.addr)
        fh.write(_object_header(self._group_messages(g)))

    # ---- deferred data
    def data_offset(self, path: str) -> int:
        """File offset of a dataset's contiguous data (after close)."""
        if not self._laid_out:
            raise H5FormatError("close() lays out the file first")
        return self._lookup(path).data_addr


# ---------------------------------------------------------------------------
#  Reader
# ---------------------------------------------------------------------------
class H5Object:
    def __init__(self, f: "H5Reader", addr: int):
        self.f, self.addr = f, addr
        self.messages = f._header_messages(addr)
        self.attrs = {}
        for t, body in self.messages:
            if t == MSG_ATTRIBUTE:
                name, val = f._decode_attribute(body)
                self.attrs[name] = val


class H5Group(H5Object):
    def __init__(self, f, addr):
        super().__init__(f, addr)
        stab = [b for t, b in self.messages if t == MSG_STAB]
        if not stab:
            raise H5FormatError("group without a symbol table (new-style groups are not supported)")
        self.tree_addr, self.heap_addr = struct.unpack_from("<QQ", stab[0])
        self.links = f._group_links(self.tree_addr, self.heap_addr)

    def keys(self):
        return list(self.links)

    def __getitem__(self, path: str):
        obj = self
        for p in [p for p in path.strip("/").split("/") if p]:
            if not isinstance(obj, H5Group) or p not in obj.links:
                raise KeyError(path)
            obj = obj.f._object(obj.links[p])
        return obj

    def __contains__(self, path: str) -> bool:
        try:
            self[path]
            return True
        except KeyError:
            return False


class H5Dataset(H5Object):
    def __init__(self, f, addr):
        super().__init__(f, addr)
        kinds = {t: b for t, b in self.messages}
        if MSG_DATASPACE not in kinds or MSG_DATATYPE not in kinds or MSG_LAYOUT not in kinds:
            raise H5FormatError("dataset header lacks dataspace, datatype or layout")
        self.shape = decode_dataspace(kinds[MSG_DATASPACE])
        self.dtype = decode_datatype(kinds[MSG_DATATYPE])
        self._layout(kinds[MSG_LAYOUT])

    def _layout(self, b: bytes) -> None:
        ver = b[0]
        self.compact = None
        if ver == 3:
            cls = b[1]
            if cls == 1:
                self.data_addr, self.size = struct.unpack_from("<QQ", b, 2)
            elif cls == 0:
                n = struct.unpack_from("<H", b, 2)[0]
                self.compact, self.data_addr, self.size = bytes(b[4:4 + n]), UNDEF, n
            else:
                raise H5FormatError("chunked layout is not supported")
        elif ver in (1, 2):
            rank, cls = b[1], b[2]
            if cls != 1:
                raise H5FormatError("layout class %d (version %d) is not supported" % (cls, ver))
            self.data_addr = struct.unpack_from("<Q", b, 8)[0]
            self.size = int(np.prod(self.shape, dtype=np.int64)) * self.dtype.itemsize
        else:
            raise H5FormatError("layout message version %d" % ver)

    def read(self) -> np.ndarray:
        n = int(np.prod(self.shape, dtype=np.int64))
        if self.compact is not None:
            raw = self.compact
        elif self.data_addr == UNDEF:
            raw = bytes(n * self.dtype.itemsize)   # never written: the default fill value
        else:
            raw = self.f._read(self.data_addr, n * self.dtype.itemsize)
        return np.frombuffer(raw, self.dtype, count=n).reshape(self.shape).copy()

    def read_rows(self, first: int, count: int) -> np.ndarray:
        """Rows first..first+count-1 of the slowest dimension (contiguous layout)."""
        if self.compact is not None or self.data_addr == UNDEF:
            return self.read()[first:first + count]
        row = int(np.prod(self.shape[1:], dtype=np.int64))
        raw = self.f._read(self.data_addr + first * row * self.dtype.itemsize, count * row * self.dtype.itemsize)
        return np.frombuffer(raw, self.dtype).reshape((count,) + tuple(self.shape[1:])).copy()


class H5Reader(H5Group):
    """Read access to a file of the structures listed in the module docstring."""

    def __init__(self, path: str):
        self.fh = open(path, "rb")
        self.base = self._find_superblock()
        sb = self._read_abs(self.base, 96)
        ver = sb[8]
        if ver not in (0, 1):
            raise H5FormatError("superblock version %d is not supported" % ver)
        if sb[13] != 8 or sb[14] != 8:
            raise H5FormatError("only 8-byte offsets and lengths are supported")
        off = 24 if ver == 0 else 28
        base_addr, _, self.eof, _ = struct.unpack_from("<QQQQ", sb, off)
        if base_addr != self.base:
            self.base = base_addr
        ent = off + 32
        _, root_addr = struct.unpack_from("<QQ", sb, ent)
        self.f = self
        self._cache: Dict[int, H5Object] = {}
        H5Group.__init__(self, self, root_addr)

    def close(self):
        self.fh.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _find_superblock(self) -> int:
        size = os.fstat(self.fh.fileno()).st_size
        pos = 0
        while pos + 8 <= size:
            if self._read_abs(pos, 8) == SIGNATURE:
                return pos
            pos = 512 if pos == 0 else pos * 2
        raise H5FormatError("no HDF5 superblock found")

    def _read_abs(self, pos: int, n: int) -> bytes:
        self.fh.seek(pos)
        b = self.fh.read(n)
        if len(b) != n:
            raise H5FormatError("read past the end of the file at %d" % pos)
        return b

    def _read(self, addr: int, n: int) -> bytes:
        return self._read_abs(self.base + addr, n)

    def _object(self, addr: int) -> H5Object:
        if addr not in self._cache:
            msgs = self._header_messages(addr)
            kinds = {t for t, _ in msgs}
            self._cache[addr] = H5Group(self, addr) if MSG_STAB in kinds else H5Dataset(self, addr)
        return self._cache[addr]

    def _header_messages(self, addr: int) -> List[Tuple[int, bytes]]:
        pre = self._read(addr, 16)
        if pre[:4] == b"OHDR":
            raise H5FormatError("version-2 object headers are not supported")
        ver, _, nmsg, _, size = struct.unpack_from("<BBHII", pre)
        if ver != 1:
            raise H5FormatError("object header version %d" % ver)
        chunks = [(addr + 16, size)]
        out = []
        while chunks and len(out) < nmsg:
            a, n = chunks.pop(0)
            data = self._read(a, n)
            p = 0
            while p + 8 <= n and len(out) < nmsg:
                t, sz, flags = struct.unpack_from("<HHB", data, p)
                body = data[p + 8:p + 8 + sz]
                if flags & 0x02:
                    raise H5FormatError("shared header messages are not supported")
                if t == MSG_CONTINUATION:
                    ca, cn = struct.unpack_from("<QQ", body)
                    chunks.append((ca, cn))
                out.append((t, body))
                p += 8 + sz
        return out

    def _heap_names(self, heap_addr: int) -> Tuple[bytes, int]:
        h = self._read(heap_addr, 32)
        if h[:4] != b"HEAP":
            raise H5FormatError("bad local heap signature")
        seg_size, _, seg_addr = struct.unpack_from("<QQQ", h, 8)
        return self._read(seg_addr, seg_size), seg_size

    def _group_links(self, tree_addr: int, heap_addr: int) -> Dict[str, int]:
        seg, _ = self._heap_names(heap_addr)

        def name_at(o):
            e = seg.index(b"\0", o)
            return seg[o:e].decode("ascii")

        links: Dict[str, int] = {}

        def walk(addr):
            hdr = self._read(addr, 24)
            if hdr[:4] != b"TREE" or hdr[4] != 0:
                raise H5FormatError("bad group B-tree node")
            level, used = hdr[5], struct.unpack_from("<H", hdr, 6)[0]
            body = self._read(addr + 24, used * 16 + 8)
            for i in range(used):
                child = struct.unpack_from("<Q", body, 8 + 16 * i)[0]
                if level > 0:
                    walk(child)
                    continue
                sn = self._read(child, 8)
                if sn[:4] != b"SNOD":
                    raise H5FormatError("bad symbol-table node")
                nsym = struct.unpack_from("<H", sn, 6)[0]
                ents = self._read(child + 8, nsym * ENTRY_SIZE)
                for j in range(nsym):
                    noff, oaddr = struct.unpack_from("<QQ", ents, j * ENTRY_SIZE)
                    links[name_at(noff)] = oaddr

        walk(tree_addr)
        return links

    def _decode_attribute(self, b: bytes):
        ver = b[0]
        if ver != 1:
            raise H5FormatError("attribute message version %d is not supported" % ver)
        nlen, tlen, slen = struct.unpack_from("<HHH", b, 2)
        p = 8
        name = b[p:p + nlen].split(b"\0")[0].decode("ascii")
        p += _pad8(nlen)
        dt = decode_datatype(b[p:p + tlen])
        p += _pad8(tlen)
        shape = decode_dataspace(b[p:p + slen])
        p += _pad8(slen)
        n = int(np.prod(shape, dtype=np.int64))
        return name, np.frombuffer(b[p:p + n * dt.itemsize], dt, count=n).reshape(shape).copy()
