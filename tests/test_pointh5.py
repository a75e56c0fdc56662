"""point/point.h5 without libhdf5: the reference's grid file
(src_mpi_primal/point_preprocessor.F90:177-546) written in the classic HDF5
layout and read back, a file in the newer layout (version 2 superblock and
object headers, link messages, version 3 attributes) read, and broken files
rejected with PointH5Error."""
import struct

import numpy as np
import pytest

from mfcfd_b200 import pointh5 as P
from mfcfd_b200.grid import naca_ogrid

FIELDS = ("x", "y", "nx", "ny", "min_dist", "flag_1", "flag_2", "left", "right", "nbhs", "conn",
          "original_id", "qtdepth")


def test_grid_round_trip(tmp_path):
    g = naca_ogrid(48, 20, seed=3, first_spacing=5e-3)
    path = str(tmp_path / "point" / "point.h5")
    P.write_grid_h5(g, path)
    g2 = P.read_grid_h5(path)
    for k in FIELDS:
        assert np.array_equal(getattr(g, k), getattr(g2, k)), k
    d = P.read_point_h5(path, 0)
    assert (d["total"], d["local"], d["ghost"]) == (g.n, g.n, 0)
    # columns as the reference reads them: id, x, y, nx, ny, min_dist, left,
    # right, qtdepth, flag_1, flag_2, nbhs, conn...
    rows = d["local_rows"]
    assert rows.shape == (g.n, 12 + int(g.nbhs.max()))
    k = 77
    assert rows[k, 1] == g.x[k] and rows[k, 5] == g.min_dist[k] and rows[k, 9] == g.flag_1[k]
    assert list(rows[k, 12:12 + g.nbhs[k]]) == list(g.conn[:g.nbhs[k], k])


def test_written_file_structure(tmp_path):
    """Fields a reader of the classic layout checks: superblock version 0 with
    8-byte offsets and lengths, the end-of-file address equal to the file
    size, the root symbol table entry caching its B-tree and heap, and the
    signatures of every structure they point to."""
    g = naca_ogrid(16, 6, seed=1, first_spacing=5e-3)
    path = str(tmp_path / "p.h5")
    P.write_grid_h5(g, path)
    data = open(path, "rb").read()
    assert data[:8] == P.SIGNATURE
    assert data[8] == 0 and data[13] == 8 and data[14] == 8
    leaf_k, int_k = struct.unpack_from("<HH", data, 16)
    assert (leaf_k, int_k) == (P.LEAF_K, P.INTERNAL_K)
    base, free, eof, drv = struct.unpack_from("<QQQQ", data, 24)
    assert base == 0 and free == P.UNDEF and drv == P.UNDEF and eof == len(data)
    name_off, oh, cache, _, tree, heap = struct.unpack_from("<QQIIQQ", data, 56)
    assert name_off == 0 and cache == 1
    assert data[oh] == 1 and data[tree:tree + 4] == b"TREE" and data[heap:heap + 4] == b"HEAP"
    assert all(a % 8 == 0 for a in (oh, tree, heap))
    # the root B-tree's one child is a symbol table node holding "1"
    child = struct.unpack_from("<Q", data, tree + 24 + 8)[0]
    assert data[child:child + 4] == b"SNOD" and struct.unpack_from("<H", data, child + 6)[0] == 1


def test_multi_rank_groups(tmp_path):
    """Twelve rank groups /1 .. /12: more names than one symbol table node
    holds, so the root B-tree has two children."""
    rng = np.random.default_rng(5)
    parts = [(rng.random((10 + r, 15)), rng.random((r, 4))) for r in range(12)]
    path = str(tmp_path / "m.h5")
    P.write_point_h5(path, parts)
    for r, (loc, gh) in enumerate(parts):
        d = P.read_point_h5(path, r)
        assert np.array_equal(d["local_rows"], loc) and np.array_equal(d["ghost_rows"], gh)
        assert (d["total"], d["local"], d["ghost"]) == (10 + 2 * r, 10 + r, r)
    with pytest.raises(P.PointH5Error, match="no object '13'"):
        P.read_point_h5(path, 12)


def test_driver_reads_point_h5_first(tmp_path):
    from mfcfd_b200 import io
    from mfcfd_b200.driver import read_case_grid
    g = naca_ogrid(24, 8, seed=2, first_spacing=5e-3)
    io.write_partgrid(naca_ogrid(24, 8, seed=9, first_spacing=5e-3),
                      str(tmp_path / "point" / "partGrid"))
    assert not np.array_equal(read_case_grid(str(tmp_path)).x, g.x)  # partGrid only
    P.write_grid_h5(g, str(tmp_path / "point" / "point.h5"))
    assert np.array_equal(read_case_grid(str(tmp_path)).x, g.x)


# --- a file in the newer layout, built by hand from the specification ------

def _ohdr(messages, cont=None):
    """Version 2 object header (4-byte chunk size, no times); `cont` =
    (address, length) appends a continuation message."""
    body = b""
    for mtype, data in messages:
        body += struct.pack("<BHB", mtype, len(data), 0) + data
    if cont is not None:
        data = struct.pack("<QQ", *cont)
        body += struct.pack("<BHB", P.MSG_CONTINUATION, len(data), 0) + data
    return b"OHDR" + struct.pack("<BBI", 2, 0x02, len(body)) + body + b"\0\0\0\0"


def _link(name, addr):
    nm = name.encode()
    return P.MSG_LINK, struct.pack("<BBB", 1, 0, len(nm)) + nm + struct.pack("<Q", addr)


def _attr_v3(name, value):
    nm = name.encode() + b"\0"
    dt = struct.pack("<BBBBI", 0x10, 0x08, 0, 0, 8) + struct.pack("<HH", 0, 64)  # int64
    ds = struct.pack("<BBBB", 2, 0, 0, 0)  # version 2, scalar
    return P.MSG_ATTRIBUTE, (struct.pack("<BBHHHB", 3, 0, len(nm), len(dt), len(ds), 0) + nm +
                             dt + ds + struct.pack("<q", value))


def _dataset_v2(addr, shape):
    ds = struct.pack("<BBBB", 2, len(shape), 0, 1) + b"".join(struct.pack("<Q", d) for d in shape)
    dt = P._dtype_f64()
    nbytes = int(np.prod(shape)) * 8
    lay = struct.pack("<BBQQ", 3, 1, addr if nbytes else P.UNDEF, nbytes)
    return [(P.MSG_DATASPACE, ds), (P.MSG_DATATYPE, dt), (P.MSG_LAYOUT, lay)]


def _new_layout_file(local, ghost):
    """Superblock v2; root, group /1 (its attributes in an OCHK continuation
    chunk) and the two datasets as version 2 object headers."""
    buf = bytearray(b"\0" * 48)
    def place(b):
        buf.extend(b"\0" * ((-len(buf)) % 8))
        off = len(buf)
        buf.extend(b)
        return off
    a_local = place(local.astype("<f8").tobytes())
    a_ghost = place(ghost.astype("<f8").tobytes())
    d_local = place(_ohdr(_dataset_v2(a_local, local.shape)))
    d_ghost = place(_ohdr(_dataset_v2(a_ghost, ghost.shape)))
    attrs = b"".join(struct.pack("<BHB", t, len(d), 0) + d for t, d in
                     (_attr_v3("total", local.shape[0] + ghost.shape[0]),
                      _attr_v3("local", local.shape[0]), _attr_v3("ghost", ghost.shape[0])))
    ochk = b"OCHK" + attrs + b"\0\0\0\0"
    a_ochk = place(ochk)
    grp = place(_ohdr([_link("local", d_local), _link("ghost", d_ghost)],
                      cont=(a_ochk, len(ochk))))
    root = place(_ohdr([_link("1", grp)]))
    sb = P.SIGNATURE + struct.pack("<BBBB", 2, 8, 8, 0)
    sb += struct.pack("<QQQQ", 0, P.UNDEF, len(buf), root) + b"\0\0\0\0"
    buf[:48] = sb
    return bytes(buf)


def test_reads_the_newer_layout(tmp_path):
    rng = np.random.default_rng(7)
    local, ghost = rng.random((9, 14)), rng.random((3, 4))
    path = tmp_path / "new.h5"
    path.write_bytes(_new_layout_file(local, ghost))
    d = P.read_point_h5(str(path), 0)
    assert (d["total"], d["local"], d["ghost"]) == (12, 9, 3)
    assert np.array_equal(d["local_rows"], local) and np.array_equal(d["ghost_rows"], ghost)


# --- broken files ------------------------------------------------------------

def test_broken_files_are_rejected(tmp_path):
    g = naca_ogrid(16, 6, seed=1, first_spacing=5e-3)
    good = tmp_path / "good.h5"
    P.write_grid_h5(g, str(good))
    data = good.read_bytes()
    cases = {
        "not_hdf5": b"this is not an HDF5 file" * 40,
        "truncated": data[: len(data) // 2],
        "bad_tree": data.replace(b"TREE", b"TRE!", 1),
        "empty": b"",
    }
    for name, blob in cases.items():
        p = tmp_path / f"{name}.h5"
        p.write_bytes(blob)
        with pytest.raises(P.PointH5Error):
            P.read_point_h5(str(p), 0)
    with pytest.raises(P.PointH5Error):
        P.read_point_h5(str(tmp_path / "missing.h5"), 0)
    # a stencil wider than the rows hold
    rows = P.grid_rows(g)
    rows[0, 11] = rows.shape[1]
    bad = tmp_path / "wide.h5"
    P.write_point_h5(str(bad), [(rows, np.zeros((0, 4)))])
    with pytest.raises(P.PointH5Error, match="nbhs out of range"):
        P.read_grid_h5(str(bad))
