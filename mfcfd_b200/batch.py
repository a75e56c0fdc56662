"""Batched runs of many grids on one GPU over the C ABI (mfcfd_batch_*).

``Batch`` holds independent instances, each a grid with its own flow
parameters, set up exactly as ``Solver`` sets up one grid.  ``run(tol,
max_iters)`` advances every instance through the reference's loop
(q_lskum.F90:59-73) until its residue is <= tol, it has run max_iters
iterations, or its residue is NaN; an instance's states and residues are
bit-identical to a ``Solver`` run of the same grid.  The reference runs one
grid per process; this has no counterpart there.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .grid import Grid
from .solver import _dptr, _ptr, make_params


@dataclass
class BatchResult:
    iters_done: np.ndarray   # [n_inst] iterations run in this call
    state: list              # [n_inst] "converged" | "max_iters" | "nonfinite"
    residue: list            # [n_inst] residue history of each instance
    status: int              # MFCFD_OK or MFCFD_ERR_NONFINITE


class Batch:
    """Device-resident batch of independent LSKUM primal problems."""

    def __init__(self, grids: list, flows: list):
        if len(grids) != len(flows):
            raise ValueError("one flow dict per grid")
        self.lib = _lib.load()
        self.grids = list(grids)
        self.n_inst = len(grids)
        params = [make_params(**f) for f in flows]
        self._params = (_lib.Params * self.n_inst)(*params)
        self._keep = []
        gstructs = []
        for g in self.grids:
            arrs = [np.ascontiguousarray(a) for a in
                    (g.x, g.y, g.nx, g.ny, g.min_dist, g.flag_1, g.flag_2, g.left, g.right,
                     g.nbhs, g.conn)]
            self._keep.append(arrs)
            gstructs.append(_lib.Grid(g.n, *[_ptr(v) for v in arrs], g.n, g.shapes))
        self._gstructs = gstructs
        ptrs = (C.POINTER(_lib.Grid) * self.n_inst)(*[C.pointer(s) for s in gstructs])
        h = C.c_void_p()
        st = self.lib.mfcfd_batch_create(self.n_inst, ptrs, self._params, C.byref(h))
        self._check(st, "mfcfd_batch_create", handle=None)
        self.h = h

    def _check(self, st, what, handle=...):
        if st == _lib.MFCFD_OK:
            return
        hh = self.h if handle is ... else handle
        detail = self.lib.mfcfd_batch_last_error(hh).decode(errors="replace")
        text = self.lib.mfcfd_strerror(st).decode()
        raise _lib.MfcfdError(st, f"{what}: {text}" + (f": {detail}" if detail else ""))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mfcfd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # state ---------------------------------------------------------------
    def set_state(self, i: int, prim: np.ndarray) -> None:
        n = self.grids[i].n
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        if prim.shape != (n, 4):
            raise ValueError(f"prim must be ({n}, 4)")
        self._check(self.lib.mfcfd_batch_set_state(self.h, int(i), _dptr(prim)),
                    "mfcfd_batch_set_state")

    def get_state(self, i: int) -> np.ndarray:
        out = np.empty((self.grids[i].n, 4))
        self._check(self.lib.mfcfd_batch_get_state(self.h, int(i), _dptr(out)),
                    "mfcfd_batch_get_state")
        return out

    # loop ----------------------------------------------------------------
    def run(self, max_iters: int, tol: float = -np.inf) -> BatchResult:
        done = np.zeros(self.n_inst, dtype=np.int32)
        state = np.zeros(self.n_inst, dtype=np.int32)
        res = np.zeros((self.n_inst, max(max_iters, 1)))
        st = self.lib.mfcfd_batch_run(self.h, float(tol), int(max_iters),
                                      done.ctypes.data_as(C.POINTER(C.c_int)),
                                      state.ctypes.data_as(C.POINTER(C.c_int)), _dptr(res))
        if st != _lib.MFCFD_ERR_NONFINITE:
            self._check(st, "mfcfd_batch_run")
        return BatchResult(done, [_lib.BATCH_STATES[int(s)] for s in state],
                           [res[i, :done[i]].copy() for i in range(self.n_inst)], st)

    def forces(self, i: int):
        g = self.grids[i]
        s = g.shapes
        cl, cd, cm = np.zeros(s), np.zeros(s), np.zeros(s)
        cp = np.zeros(int((g.flag_2 > 0).sum()))
        self._check(self.lib.mfcfd_batch_forces(self.h, int(i), _dptr(cl), _dptr(cd), _dptr(cm),
                                                _dptr(cp)), "mfcfd_batch_forces")
        return cl, cd, cm, cp

    # launch shape ----------------------------------------------------------
    def tune(self, iters: int = 4) -> float:
        ms = C.c_double(0.0)
        self._check(self.lib.mfcfd_batch_tune(self.h, int(iters), C.byref(ms)), "mfcfd_batch_tune")
        return ms.value

    def set_launch(self, point_block: int = 256, point_grid: int = 0, flux_grid: int = 0):
        self._check(self.lib.mfcfd_batch_set_launch(self.h, int(point_block), int(point_grid),
                                                    int(flux_grid)), "mfcfd_batch_set_launch")

    def set_stream(self, stream) -> None:
        self._check(self.lib.mfcfd_batch_set_stream(self.h, C.c_void_p(stream)),
                    "mfcfd_batch_set_stream")

    def info(self) -> dict:
        n, pb, pg, fg = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        npts = C.c_longlong()
        self._check(self.lib.mfcfd_batch_info(self.h, C.byref(n), C.byref(npts), C.byref(pb),
                                              C.byref(pg), C.byref(fg)), "mfcfd_batch_info")
        return {"n_inst": n.value, "n_points": npts.value, "point_block": pb.value,
                "point_grid": pg.value, "flux_grid": fg.value}

    def launch_count(self) -> int:
        return int(self.lib.mfcfd_batch_launch_count(self.h))
