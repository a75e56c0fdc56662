"""``point/point.h5``: the reference's grid file, read and written without libhdf5.

The reference reads its point cloud with the HDF5 library
(``src_mpi_primal/point_preprocessor.F90:177-546``): per rank r the group
``/<r+1>`` with three integer attributes ``total``, ``local`` and ``ghost``
(``:254-280``), the dataset ``<group>/local`` of float64 rows, one per point,
with columns id, x, y, nx, ny, min_dist, left, right, qtdepth, flag_1,
flag_2, nbhs, conn(1..nbhs) (``:353-371``; C dimensions [local][12 + Kmax],
which Fortran sees as (12 + Kmax, local)), and ``<group>/ghost`` with rows
global id, x, y, min_dist of the rank's ghost points (``:489-501``).

Neither libhdf5 nor h5py is available on these machines, so this module
implements the part of the HDF5 file format (the public "HDF5 File Format
Specification", version 3.0) that this one layout needs:

* writer: the classic layout the HDF5 library produces by default -- version 0
  superblock, version 1 object headers, groups as symbol tables (version 1
  B-tree of group nodes, symbol table nodes, local heap of link names),
  contiguous datasets (layout message version 3), scalar attributes (message
  version 1), little-endian IEEE float64 and int32;
* reader: that layout, plus what newer HDF5 writers emit for the same data --
  version 2/3 superblocks, version 2 object headers with continuation chunks,
  compact link messages, attribute messages of versions 1-3, dataspace
  messages of versions 1-2, compact and contiguous layouts, fixed-point and
  IEEE floating-point types of either byte order.  Anything else (chunked or
  filtered storage, dense link storage, shared messages, variable-length
  types) is rejected with ``PointH5Error`` naming what was found.
"""
from __future__ import annotations

import os
import struct

import numpy as np

from .grid import MAX_NBHS, Grid

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K = 4        # group leaf node K: a symbol table node holds 2K entries
INTERNAL_K = 16   # group internal node K: a B-tree node holds 2K children

# object header message types
MSG_NIL, MSG_DATASPACE, MSG_LINK_INFO, MSG_DATATYPE = 0x0, 0x1, 0x2, 0x3
MSG_FILL_OLD, MSG_FILL, MSG_LINK, MSG_LAYOUT = 0x4, 0x5, 0x6, 0x8
MSG_GROUP_INFO, MSG_FILTERS, MSG_ATTRIBUTE = 0xA, 0xB, 0xC
MSG_CONTINUATION, MSG_SYMBOL_TABLE, MSG_MTIME = 0x10, 0x11, 0x12


class PointH5Error(ValueError):
    """The file is not an HDF5 file of the point.h5 layout this module reads."""


def _pad8(n: int) -> int:
    return (n + 7) & ~7


# ---------------------------------------------------------------------------
# writer

class _File:
    """A growing byte image with 8-byte aligned allocations."""

    def __init__(self):
        self.buf = bytearray()

    def alloc(self, size: int) -> int:
        self.buf += b"\0" * ((-len(self.buf)) % 8)
        off = len(self.buf)
        self.buf += b"\0" * size
        return off

    def put(self, off: int, data: bytes) -> None:
        self.buf[off:off + len(data)] = data


def _msg(mtype: int, body: bytes, flags: int = 0) -> bytes:
    body = body + b"\0" * (_pad8(len(body)) - len(body))
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _object_header(f: _File, messages) -> int:
    """Version 1 object header holding `messages` (already encoded)."""
    data = b"".join(messages)
    off = f.alloc(16 + len(data))
    f.put(off, struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(data)) + data)
    return off


def _dtype_f64() -> bytes:
    # class 1 (floating point), version 1; little-endian, implied msb
    # normalisation, sign bit 63; offset 0, precision 64, exponent at bit 52
    # of 11 bits, mantissa at bit 0 of 52 bits, exponent bias 1023
    return struct.pack("<BBBBI", 0x11, 0x20, 63, 0, 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11,
                                                                       0, 52, 1023)


def _dtype_i32() -> bytes:
    # class 0 (fixed point), version 1; little-endian, signed; offset 0, precision 32
    return struct.pack("<BBBBI", 0x10, 0x08, 0, 0, 4) + struct.pack("<HH", 0, 32)


def _dataspace_v1(dims) -> bytes:
    body = struct.pack("<BBB5x", 1, len(dims), 0)
    return body + b"".join(struct.pack("<Q", int(d)) for d in dims)


def _attribute_i32(name: str, value: int) -> bytes:
    nm = name.encode("ascii") + b"\0"
    dt, ds = _dtype_i32(), _dataspace_v1(())
    body = struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(ds))
    body += nm + b"\0" * (_pad8(len(nm)) - len(nm))
    body += dt + b"\0" * (_pad8(len(dt)) - len(dt))
    body += ds + b"\0" * (_pad8(len(ds)) - len(ds))
    body += struct.pack("<i", int(value))
    return _msg(MSG_ATTRIBUTE, body)


def _dataset(f: _File, array: np.ndarray) -> int:
    a = np.ascontiguousarray(array, dtype="<f8")
    if a.size:
        data_off = f.alloc(a.nbytes)
        f.put(data_off, a.tobytes())
    else:
        data_off = UNDEF
    msgs = [
        _msg(MSG_DATASPACE, _dataspace_v1(a.shape)),
        _msg(MSG_DATATYPE, _dtype_f64(), flags=1),  # constant
        # fill value v2: allocation time late, write time "if set", no value
        _msg(MSG_FILL, struct.pack("<BBBB", 2, 2, 2, 0), flags=1),
        _msg(MSG_LAYOUT, struct.pack("<BBQQ", 3, 1, data_off, a.nbytes)),
    ]
    return _object_header(f, msgs)


def _group(f: _File, entries, attributes=()):
    """A symbol-table group over `entries` = [(name, object header address,
    (btree, heap) or None)].  Returns (object header, B-tree, heap) addresses."""
    entries = sorted(entries, key=lambda e: e[0].encode())
    # local heap: "" at offset 0, then each name, null-terminated, padded to 8
    names = bytearray(b"\0" * 8)
    offs = {}
    for name, _, _ in entries:
        offs[name] = len(names)
        nm = name.encode("ascii") + b"\0"
        names += nm + b"\0" * (_pad8(len(nm)) - len(nm))
    heap = f.alloc(32)
    heap_data = f.alloc(len(names))
    f.put(heap_data, bytes(names))
    f.put(heap, b"HEAP" + struct.pack("<B3xQQQ", 0, len(names), UNDEF, heap_data))
    # symbol table nodes of at most 2*LEAF_K entries, one B-tree leaf over them
    cap = 2 * LEAF_K
    chunks = [entries[i:i + cap] for i in range(0, len(entries), cap)] or [[]]
    if len(chunks) > 2 * INTERNAL_K:
        raise PointH5Error(f"more than {2 * INTERNAL_K * cap} links in one group")
    snods = []
    for chunk in chunks:
        node = f.alloc(8 + cap * 40)
        body = b"SNOD" + struct.pack("<BBH", 1, 0, len(chunk))
        for name, oh, cache in chunk:
            if cache is None:
                body += struct.pack("<QQII16x", offs[name], oh, 0, 0)
            else:
                body += struct.pack("<QQIIQQ", offs[name], oh, 1, 0, cache[0], cache[1])
        f.put(node, body)
        snods.append((node, chunk[-1][0] if chunk else None))
    tree = f.alloc(24 + 2 * INTERNAL_K * 8 + (2 * INTERNAL_K + 1) * 8)
    nused = len(snods) if entries else 0
    body = b"TREE" + struct.pack("<BBHQQ", 0, 0, nused, UNDEF, UNDEF)
    body += struct.pack("<Q", 0)  # key 0: the empty name
    for node, last in snods[:nused]:
        body += struct.pack("<QQ", node, offs[last])
    f.put(tree, body)
    msgs = [_msg(MSG_SYMBOL_TABLE, struct.pack("<QQ", tree, heap))]
    msgs += [_attribute_i32(n, v) for n, v in attributes]
    oh = _object_header(f, msgs)
    return oh, tree, heap


def write_point_h5(path: str, parts) -> None:
    """Writes ``parts`` = [(local rows (L, W) float64, ghost rows (G, 4)
    float64), ...] as groups /1, /2, ... of a point.h5 file."""
    f = _File()
    sb = f.alloc(96)
    groups = []
    for r, (local, ghost) in enumerate(parts):
        local = np.asarray(local, dtype=np.float64)
        ghost = np.asarray(ghost, dtype=np.float64).reshape(-1, 4)
        if local.ndim != 2 or local.shape[1] < 12:
            raise PointH5Error("local rows must be (points, 12 + Kmax)")
        d_local = _dataset(f, local)
        d_ghost = _dataset(f, ghost)
        nl, ng = local.shape[0], ghost.shape[0]
        oh, tree, heap = _group(f, [("local", d_local, None), ("ghost", d_ghost, None)],
                                attributes=(("total", nl + ng), ("local", nl), ("ghost", ng)))
        groups.append((str(r + 1), oh, (tree, heap)))
    root_oh, root_tree, root_heap = _group(f, groups)
    eof = len(f.buf)
    body = SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, LEAF_K, INTERNAL_K, 0)
    body += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
    body += struct.pack("<QQIIQQ", 0, root_oh, 1, 0, root_tree, root_heap)
    f.put(sb, body)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "wb") as fh:
        fh.write(bytes(f.buf))


# ---------------------------------------------------------------------------
# reader

class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        base = self._find_superblock()
        self.base = base
        v = data[base + 8]
        if v in (0, 1):
            self.so, self.sl = data[base + 13], data[base + 14]
            self.leaf_k, self.int_k = struct.unpack_from("<HH", data, base + 16)
            p = base + 24 + (4 if v == 1 else 0)
            self._check_sizes()
            base_addr, _, eof, _ = (self.uint(p + i * self.so, self.so) for i in range(4))
            p += 4 * self.so
            self.root = self.uint(p + self.so, self.so)  # symbol table entry: object header
        elif v in (2, 3):
            self.so, self.sl = data[base + 9], data[base + 10]
            self._check_sizes()
            p = base + 12
            base_addr, _, eof, root = (self.uint(p + i * self.so, self.so) for i in range(4))
            self.root = root
        else:
            raise PointH5Error(f"superblock version {v} is not supported")
        self.addr0 = base_addr if base_addr != UNDEF else 0
        if eof != UNDEF and self.addr0 + eof > len(data):
            raise PointH5Error(f"truncated file: {len(data)} bytes, the superblock says "
                               f"{self.addr0 + eof}")

    def _find_superblock(self) -> int:
        off = 0
        while off + 8 <= len(self.d):
            if self.d[off:off + 8] == SIGNATURE:
                return off
            off = 512 if off == 0 else off * 2
        raise PointH5Error("no HDF5 signature: not an HDF5 file")

    def _check_sizes(self):
        if self.so not in (4, 8) or self.sl not in (4, 8):
            raise PointH5Error(f"unsupported offset/length sizes {self.so}/{self.sl}")

    def uint(self, off: int, size: int) -> int:
        if off < 0 or off + size > len(self.d):
            raise PointH5Error(f"read past the end of the file at {off}")
        return int.from_bytes(self.d[off:off + size], "little")

    def addr(self, a: int) -> int:
        return self.addr0 + a

    def bytes_at(self, off: int, n: int) -> bytes:
        if off < 0 or off + n > len(self.d):
            raise PointH5Error(f"read past the end of the file at {off}")
        return self.d[off:off + n]

    # object headers -------------------------------------------------------
    def messages(self, oh: int):
        """[(type, flags, body)] of the object header at file address oh."""
        p = self.addr(oh)
        out = []
        if self.bytes_at(p, 4) == b"OHDR":
            self._messages_v2(p, out)
        elif self.d[p] == 1:
            nmsg = struct.unpack_from("<H", self.d, p + 2)[0]
            size = struct.unpack_from("<I", self.d, p + 8)[0]
            blocks = [(p + 16, size)]
            while blocks and len(out) < nmsg:
                start, length = blocks.pop(0)
                q, end = start, start + length
                while q + 8 <= end and len(out) < nmsg:
                    mtype, msize, mflags = struct.unpack_from("<HHB", self.d, q)
                    body = self.bytes_at(q + 8, msize)
                    q += 8 + msize
                    if mtype == MSG_CONTINUATION:
                        blocks.append((self.addr(self.uint_b(body, 0, self.so)),
                                       self.uint_b(body, self.so, self.sl)))
                    out.append((mtype, mflags, body))
        else:
            raise PointH5Error(f"unknown object header at {oh}")
        for mtype, mflags, _ in out:
            if mflags & 0x2 and mtype != MSG_NIL:
                raise PointH5Error(f"shared message of type {mtype:#x} is not supported")
        return out

    def _messages_v2(self, p: int, out):
        if self.d[p + 4] != 2:
            raise PointH5Error("object header version 2 expected")
        flags = self.d[p + 5]
        q = p + 6
        if flags & 0x20:
            q += 16  # times
        if flags & 0x10:
            q += 4   # attribute phase change values
        csize = 1 << (flags & 0x3)
        size = self.uint(q, csize)
        q += csize
        chunks = [(q, q + size)]
        head = 4 + (2 if flags & 0x4 else 0)  # message header (with creation order)
        while chunks:
            q, end = chunks.pop(0)
            while end - q >= head:  # a shorter remainder is the chunk's gap
                mtype = self.d[q]
                msize = struct.unpack_from("<H", self.d, q + 1)[0]
                mflags = self.d[q + 3]
                q += 4 + (2 if flags & 0x4 else 0)
                body = self.bytes_at(q, msize)
                q += msize
                if mtype == MSG_CONTINUATION:
                    ca = self.addr(self.uint_b(body, 0, self.so))
                    cl = self.uint_b(body, self.so, self.sl)
                    if self.bytes_at(ca, 4) != b"OCHK":
                        raise PointH5Error("bad object header continuation chunk")
                    chunks.append((ca + 4, ca + cl - 4))
                out.append((mtype, mflags, body))

    # groups -------------------------------------------------------------
    def links(self, oh: int) -> dict:
        """name -> object header address of the group at oh."""
        links = {}
        for mtype, _, body in self.messages(oh):
            if mtype == MSG_SYMBOL_TABLE:
                tree = self.uint_b(body, 0, self.so)
                heap = self.uint_b(body, self.so, self.so)
                self._walk_btree(self.addr(tree), self._heap_data(heap), links)
            elif mtype == MSG_LINK:
                name, target = self._link(body)
                if target is not None:
                    links[name] = target
            elif mtype == MSG_LINK_INFO:
                fheap = self.uint_b(body, 2 + (8 if body[1] & 1 else 0), self.so)
                if fheap != UNDEF:
                    raise PointH5Error("dense link storage (fractal heap) is not supported")
        return links

    def uint_b(self, body: bytes, off: int, size: int) -> int:
        return int.from_bytes(body[off:off + size], "little")

    def _heap_data(self, heap: int):
        p = self.addr(heap)
        if self.bytes_at(p, 4) != b"HEAP":
            raise PointH5Error("bad local heap signature")
        size = self.uint(p + 8, self.sl)
        data_addr = self.uint(p + 8 + 2 * self.sl, self.so)
        return self.bytes_at(self.addr(data_addr), size)

    def _walk_btree(self, p: int, heap: bytes, links: dict, depth: int = 0):
        if depth > 32 or self.bytes_at(p, 4) != b"TREE":
            raise PointH5Error("bad group B-tree node")
        ntype, level = self.d[p + 4], self.d[p + 5]
        used = struct.unpack_from("<H", self.d, p + 6)[0]
        if ntype != 0:
            raise PointH5Error("group B-tree of the wrong node type")
        q = p + 8 + 2 * self.so + self.sl  # past the siblings and key 0
        for _ in range(used):
            child = self.addr(self.uint(q, self.so))
            q += self.so + self.sl
            if level > 0:
                self._walk_btree(child, heap, links, depth + 1)
            else:
                self._read_snod(child, heap, links)

    def _read_snod(self, p: int, heap: bytes, links: dict):
        if self.bytes_at(p, 4) != b"SNOD":
            raise PointH5Error("bad symbol table node")
        n = struct.unpack_from("<H", self.d, p + 6)[0]
        q = p + 8
        for _ in range(n):
            name_off = self.uint(q, self.so)
            oh = self.uint(q + self.so, self.so)
            end = heap.find(b"\0", name_off)
            if end < 0:
                raise PointH5Error("link name runs past its heap")
            links[heap[name_off:end].decode("utf-8")] = oh
            q += 2 * self.so + 8 + 16

    def _link(self, body: bytes):
        if body[0] != 1:
            raise PointH5Error(f"link message version {body[0]}")
        flags = body[1]
        q = 2
        ltype = 0
        if flags & 0x8:
            ltype = body[q]
            q += 1
        if flags & 0x4:
            q += 8
        if flags & 0x10:
            q += 1
        lsize = 1 << (flags & 0x3)
        nlen = int.from_bytes(body[q:q + lsize], "little")
        q += lsize
        name = body[q:q + nlen].decode("utf-8")
        q += nlen
        if ltype != 0:
            return name, None  # soft / external links are not followed
        return name, int.from_bytes(body[q:q + self.so], "little")

    # datatypes, dataspaces, data ----------------------------------------
    def _dtype(self, body: bytes):
        cls, version = body[0] & 0x0F, body[0] >> 4
        bits0 = body[1]
        size = struct.unpack_from("<I", body, 4)[0]
        order = ">" if bits0 & 1 else "<"
        if cls == 0 and size in (1, 2, 4, 8):
            kind = "i" if bits0 & 0x08 else "u"
            return np.dtype(f"{order}{kind}{size}")
        if cls == 1 and size in (4, 8):
            return np.dtype(f"{order}f{size}")
        raise PointH5Error(f"datatype class {cls} (version {version}) of {size} bytes is not "
                           f"supported")

    def _dspace(self, body: bytes):
        version, rank, flags = body[0], body[1], body[2]
        if version == 1:
            q = 8
        elif version == 2:
            if body[3] == 2:
                return None  # null dataspace
            q = 4
        else:
            raise PointH5Error(f"dataspace message version {version}")
        return tuple(int.from_bytes(body[q + i * self.sl:q + (i + 1) * self.sl], "little")
                     for i in range(rank))

    def attributes(self, oh: int) -> dict:
        out = {}
        for mtype, _, body in self.messages(oh):
            if mtype != MSG_ATTRIBUTE:
                continue
            version = body[0]
            nsize, tsize, ssize = struct.unpack_from("<HHH", body, 2)
            if version == 1:
                q = 8
                name = body[q:q + nsize].split(b"\0")[0].decode("utf-8")
                q += _pad8(nsize)
                dt = self._dtype(body[q:q + tsize]); q += _pad8(tsize)
                dims = self._dspace(body[q:q + ssize]); q += _pad8(ssize)
            elif version in (2, 3):
                q = 8 + (1 if version == 3 else 0)
                name = body[q:q + nsize].split(b"\0")[0].decode("utf-8")
                q += nsize
                dt = self._dtype(body[q:q + tsize]); q += tsize
                dims = self._dspace(body[q:q + ssize]); q += ssize
            else:
                raise PointH5Error(f"attribute message version {version}")
            count = int(np.prod(dims)) if dims else 1
            raw = body[q:q + count * dt.itemsize]
            if len(raw) != count * dt.itemsize:
                raise PointH5Error(f"attribute {name!r} is truncated")
            val = np.frombuffer(raw, dtype=dt)
            out[name] = val.reshape(dims) if dims else val[0]
        return out

    def dataset(self, oh: int) -> np.ndarray:
        dims = dt = layout = None
        for mtype, _, body in self.messages(oh):
            if mtype == MSG_DATASPACE:
                dims = self._dspace(body)
            elif mtype == MSG_DATATYPE:
                dt = self._dtype(body)
            elif mtype == MSG_LAYOUT:
                layout = body
            elif mtype == MSG_FILTERS:
                raise PointH5Error("filtered (compressed) datasets are not supported")
        if dims is None or dt is None or layout is None:
            raise PointH5Error("dataset without dataspace, datatype or layout")
        count = int(np.prod(dims)) if dims else 1
        nbytes = count * dt.itemsize
        if layout[0] != 3:
            raise PointH5Error(f"data layout message version {layout[0]} is not supported")
        cls = layout[1]
        if cls == 0:  # compact
            size = struct.unpack_from("<H", layout, 2)[0]
            raw = layout[4:4 + size]
        elif cls == 1:  # contiguous
            a = self.uint_b(layout, 2, self.so)
            if nbytes == 0:
                raw = b""
            elif a == UNDEF:
                raw = b"\0" * nbytes  # never written: the fill value (0)
            else:
                raw = self.bytes_at(self.addr(a), nbytes)
        else:
            raise PointH5Error("chunked datasets are not supported")
        if len(raw) < nbytes:
            raise PointH5Error("dataset is truncated")
        return np.frombuffer(raw[:nbytes], dtype=dt).astype(dt.newbyteorder("=")).reshape(dims)

    def lookup(self, path: str) -> int:
        oh = self.root
        for part in [p for p in path.split("/") if p]:
            links = self.links(oh)
            if part not in links:
                raise PointH5Error(f"no object {part!r} on the path {path!r}")
            oh = links[part]
        return oh


def read_point_h5(path: str, rank: int = 0) -> dict:
    """Group ``/<rank+1>`` of a point.h5 file: {'total', 'local', 'ghost'
    (attribute values), 'local_rows' (local, W) float64, 'ghost_rows' (ghost,
    4) float64}, checked against the attributes."""
    try:
        with open(path, "rb") as fh:
            data = fh.read()
    except OSError as e:
        raise PointH5Error(f"{path}: {e}") from e
    r = _Reader(data)
    group = r.lookup(str(rank + 1))
    attrs = r.attributes(group)
    for key in ("total", "local", "ghost"):
        if key not in attrs:
            raise PointH5Error(f"{path}: group /{rank + 1} has no {key!r} attribute")
    links = r.links(group)
    for key in ("local", "ghost"):
        if key not in links:
            raise PointH5Error(f"{path}: no dataset /{rank + 1}/{key}")
    local = r.dataset(links["local"]).astype(np.float64)
    ghost = r.dataset(links["ghost"]).astype(np.float64)
    nl, ng, nt = int(attrs["local"]), int(attrs["ghost"]), int(attrs["total"])
    if local.ndim != 2 or local.shape[0] != nl or local.shape[1] < 12:
        raise PointH5Error(f"{path}: /{rank + 1}/local is {local.shape}, expected ({nl}, >= 12)")
    if ghost.size == 0:
        ghost = ghost.reshape(0, 4)
    if ghost.ndim != 2 or ghost.shape[0] < ng or ghost.shape[1] < 4:
        raise PointH5Error(f"{path}: /{rank + 1}/ghost is {ghost.shape}, expected ({ng}, 4)")
    if nt != nl + ng:
        raise PointH5Error(f"{path}: total {nt} != local {nl} + ghost {ng}")
    return {"total": nt, "local": nl, "ghost": ng, "local_rows": local,
            "ghost_rows": ghost[:ng]}


def grid_rows(grid: Grid, kmax: int | None = None) -> np.ndarray:
    """The ``local`` dataset rows of a grid (point_preprocessor.F90:353-371)."""
    n = grid.n
    kmax = int(grid.nbhs.max(initial=0)) if kmax is None else kmax
    rows = np.zeros((n, 12 + kmax))
    rows[:, 0] = grid.original_id
    rows[:, 1] = grid.x
    rows[:, 2] = grid.y
    rows[:, 3] = grid.nx
    rows[:, 4] = grid.ny
    rows[:, 5] = grid.min_dist
    rows[:, 6] = grid.left
    rows[:, 7] = grid.right
    rows[:, 8] = grid.qtdepth
    rows[:, 9] = grid.flag_1
    rows[:, 10] = grid.flag_2
    rows[:, 11] = grid.nbhs
    slot = np.arange(kmax)[:, None] < grid.nbhs[None, :]
    rows[:, 12:] = np.where(slot, grid.conn[:kmax], 0).T
    return rows


def grid_from_rows(rows: np.ndarray, shapes: int = 1, name: str = "") -> Grid:
    """A Grid from ``local`` rows, as the reference's reader assigns them
    (reals to integers by truncation, like Fortran's assignment)."""
    n, w = rows.shape
    nb = rows[:, 11].astype(np.int32)
    if n and (nb.min() < 0 or nb.max() > min(MAX_NBHS, w - 12)):
        raise PointH5Error(f"nbhs out of range [0, {min(MAX_NBHS, w - 12)}]")
    conn = np.zeros((MAX_NBHS, n), np.int32)
    k = min(MAX_NBHS, w - 12)
    slot = np.arange(k)[:, None] < nb[None, :]
    conn[:k] = np.where(slot, rows[:, 12:12 + k].T.astype(np.int32), 0)
    g = Grid(x=rows[:, 1].copy(), y=rows[:, 2].copy(), nx=rows[:, 3].copy(),
             ny=rows[:, 4].copy(), min_dist=rows[:, 5].copy(),
             flag_1=rows[:, 9].astype(np.int32), flag_2=rows[:, 10].astype(np.int32),
             left=rows[:, 6].astype(np.int32), right=rows[:, 7].astype(np.int32), nbhs=nb,
             conn=conn, original_id=rows[:, 0].astype(np.int32),
             qtdepth=rows[:, 8].astype(np.int32), shapes=shapes, name=name)
    g.validate()
    return g


def write_grid_h5(grid: Grid, path: str) -> None:
    """One-rank point.h5 of a grid: group /1, no ghost points."""
    write_point_h5(path, [(grid_rows(grid), np.zeros((0, 4)))])


def read_grid_h5(path: str, shapes: int = 1) -> Grid:
    """The grid of a one-rank point.h5 file (group /1)."""
    d = read_point_h5(path, 0)
    if d["ghost"]:
        raise PointH5Error(f"{path}: group /1 has {d['ghost']} ghost points; a one-rank grid "
                           f"has none")
    return grid_from_rows(d["local_rows"], shapes=shapes, name=os.path.basename(path))
