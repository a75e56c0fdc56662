"""CPU tests of the C ABI boundary: the library builds, loads, exports every
declared symbol, and rejects bad input before touching a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from mfcfd_b200 import _lib
from mfcfd_b200.grid import naca_ogrid
from mfcfd_b200.solver import _ptr, make_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mfcfd_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z ]+\*?\s*\*?(mfcfd_[a-z0-9_]+)\s*\(", text,
                                 re.M)))


def test_header_declares_the_bound_symbols():
    names = declared_functions()
    assert set(names) == set(_lib.EXPORTS), names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_strerror_and_defaults():
    lib = _lib.load()
    for code in range(-8, 1):
        assert lib.mfcfd_strerror(code)
    p = _lib.Params()
    assert lib.mfcfd_default_params(C.byref(p)) == 0
    assert p.rks == 4 and p.euler == 1.0 and p.vl_const == 150.0


def _create(grid, **kw):
    lib = _lib.load()
    arrays = [np.ascontiguousarray(a) for a in (grid.x, grid.y, grid.nx, grid.ny, grid.min_dist,
                                                grid.flag_1, grid.flag_2, grid.left, grid.right,
                                                grid.nbhs, grid.conn)]
    g = _lib.Grid(grid.n, *[_ptr(a) for a in arrays], grid.n, grid.shapes)
    params = make_params(cfl=0.2, **kw)
    h = C.c_void_p()
    st = lib.mfcfd_create(C.byref(g), C.byref(params), C.byref(h))
    msg = lib.mfcfd_last_error(None).decode()
    if st == 0:
        lib.mfcfd_destroy(h)
    return st, msg


def test_null_arguments_rejected():
    lib = _lib.load()
    assert lib.mfcfd_create(None, None, None) == _lib.MFCFD_ERR_ARG
    assert lib.mfcfd_run(None, 1, 1, None, None) == _lib.MFCFD_ERR_ARG
    assert lib.mfcfd_destroy(None) == 0


def test_bad_connectivity_rejected():
    g = naca_ogrid(24, 8, seed=1)
    g.conn[0, 50] = g.n + 5
    st, msg = _create(g)
    assert st == _lib.MFCFD_ERR_GRID and "conn" in msg


def test_bad_shape_flag_rejected():
    g = naca_ogrid(24, 8, seed=1)
    g.flag_2[3] = 2
    st, msg = _create(g)
    assert st == _lib.MFCFD_ERR_GRID and "shapes" in msg


def test_empty_split_list_rejected():
    """A wall point whose neighbours all lie on one side has an empty x
    list: the reference warns and then divides by zero; the library refuses."""
    g = naca_ogrid(24, 8, seed=1)
    p = 5  # wall point; keep only its left ring neighbour
    g.conn[:, p] = 0
    g.conn[0, p] = g.left[p]
    g.nbhs[p] = 1
    st, msg = _create(g)
    assert st == _lib.MFCFD_ERR_GRID and "empty split list" in msg


def test_bad_params_rejected():
    g = naca_ogrid(24, 8, seed=1)
    st, _ = _create(g, tscheme="ssprk43", inner_iterations=-1)
    assert st == _lib.MFCFD_ERR_ARG


def test_create_without_device_reports_nodev():
    from tests.conftest import have_gpu
    if have_gpu():
        pytest.skip("a CUDA device is present")
    st, msg = _create(naca_ogrid(24, 8, seed=1))
    assert st == _lib.MFCFD_ERR_NODEV
