"""CPU tests of the batched C ABI's host half: argument and grid checks run
before any device call, and the batched workload's draws."""
import ctypes as C

import numpy as np

from mfcfd_b200 import _lib
from mfcfd_b200.grid import batch_instances, naca_ogrid
from mfcfd_b200.solver import _ptr, make_params


def _create(grids, flows):
    lib = _lib.load()
    keep, structs = [], []
    for g in grids:
        arrs = [np.ascontiguousarray(a) for a in (g.x, g.y, g.nx, g.ny, g.min_dist, g.flag_1,
                                                  g.flag_2, g.left, g.right, g.nbhs, g.conn)]
        keep.append(arrs)
        structs.append(_lib.Grid(g.n, *[_ptr(a) for a in arrs], g.n, g.shapes))
    ptrs = (C.POINTER(_lib.Grid) * len(grids))(*[C.pointer(s) for s in structs])
    params = (_lib.Params * len(grids))(*[make_params(**f) for f in flows])
    h = C.c_void_p()
    st = lib.mfcfd_batch_create(len(grids), ptrs, params, C.byref(h))
    msg = lib.mfcfd_batch_last_error(None).decode()
    if st == 0:
        lib.mfcfd_batch_destroy(h)
    return st, msg


FLOW = dict(cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0)


def test_instance_count_checked():
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.mfcfd_batch_create(0, None, None, C.byref(h)) == _lib.MFCFD_ERR_ARG
    assert lib.mfcfd_batch_create(_lib.MFCFD_BATCH_MAX + 1, None, None,
                                  C.byref(h)) == _lib.MFCFD_ERR_ARG
    assert lib.mfcfd_batch_create(1, None, None, None) == _lib.MFCFD_ERR_ARG
    assert lib.mfcfd_batch_destroy(None) == 0
    assert lib.mfcfd_batch_run(None, 0.0, 1, None, None, None) == _lib.MFCFD_ERR_ARG


def test_shared_parameters_must_agree():
    g = naca_ogrid(24, 8, seed=1)
    st, msg = _create([g, g], [FLOW, dict(FLOW, cfl=0.3)])
    assert st == _lib.MFCFD_ERR_ARG and "params[1]" in msg
    st, msg = _create([g, g], [FLOW, dict(FLOW, inner_iterations=2)])
    assert st == _lib.MFCFD_ERR_ARG


def test_bad_grid_is_named_by_instance():
    good = naca_ogrid(24, 8, seed=1)
    bad = naca_ogrid(24, 8, seed=2)
    bad.conn[0, 30] = bad.n + 3
    st, msg = _create([good, good, bad], [FLOW, dict(FLOW, mach=0.7), FLOW])
    assert st == _lib.MFCFD_ERR_GRID and msg.startswith("instance 2:") and "conn" in msg


def test_valid_batch_reaches_the_device_check():
    g1, g2 = naca_ogrid(24, 8, seed=1), naca_ogrid(32, 10, seed=2)
    st, msg = _create([g1, g2], [FLOW, dict(FLOW, mach=0.7, aoa=-1.0, vl_const=3.0)])
    import torch
    if not torch.cuda.is_available():
        assert st == _lib.MFCFD_ERR_NODEV, msg
    else:
        assert st == _lib.MFCFD_OK, msg


def test_batch_draws():
    _, flows, specs = batch_instances(64, build=False)
    n = np.array([s["ni"] * s["nj"] for s in specs])
    assert n.min() >= 0.9 * 4000 and n.max() <= 1.1 * 256000
    assert all(0.5 <= f["mach"] <= 0.8 and -2.0 <= f["aoa"] <= 4.0 for f in flows)
    assert all(0.08 <= s["thickness"] <= 0.16 for s in specs)
    assert all(s["ni"] % 2 == 0 and abs(s["ni"] / s["nj"] - 1.6) < 0.1 for s in specs)
    _, _, again = batch_instances(64, build=False)
    assert again == specs
