"""Host-side mirror of the reference's primal loop over the C ABI.

``Solver`` holds one device-resident problem (one ``mfcfd_t`` handle); its
methods follow the reference's call sequence in
src_mpi_primal/meshfree_solver.F90:83 -> q_lskum.F90:16-79:

* construction = read grid + allocate_soln + initial_conditions +
  compute_normals + generate_connectivity,
* ``run(n)`` = ``n`` passes of the ``do it = itr+1, itr+max_iters`` loop with
  fpi_solver, returning the residue history (the loop stops at a NaN residue,
  as q_lskum.F90:71 does),
* ``forces()`` = compute_cl_cd_cm (Cl, Cd, Cm per shape, cp per shape point).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .grid import Grid

_PREC = {"fp64": _lib.MFCFD_FP64, "fp32_mixed": _lib.MFCFD_FP32_MIXED}
_ORDER = {"kind": _lib.MFCFD_ORDER_KIND, "rcm": _lib.MFCFD_ORDER_RCM}


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_params(cfl=0.2, power=0.0, vl_const=150.0, mach=0.63, aoa=2.0, tscheme="ssprk43",
                inner_iterations=0, interior_points_normal_flag=0, format=1, restart=0,
                res_old=0.0, precision="fp64", ordering="kind") -> _lib.Params:
    """Case parameters with the reference's readcase defaults (readcase.F90)."""
    if tscheme == "ssprk43":
        rks, euler = 4, 1.0
    elif tscheme == "first":
        rks, euler = 1, 2.0
    else:
        raise ValueError(f"unknown tscheme {tscheme!r}")
    return _lib.Params(cfl, power, vl_const, mach, aoa, rks, euler, inner_iterations,
                       interior_points_normal_flag, format, restart, res_old,
                       _PREC[precision], _ORDER[ordering])


class Solver:
    """Device-resident LSKUM primal solver for one grid (FP64 path)."""

    def __init__(self, grid: Grid, **params):
        self.lib = _lib.load()
        self.grid = grid
        self.n = grid.n
        self.params = make_params(**params)
        self.it = 0 if self.params.restart == 0 else None
        g = grid
        self._arrays = [np.ascontiguousarray(a) for a in
                        (g.x, g.y, g.nx, g.ny, g.min_dist, g.flag_1, g.flag_2, g.left, g.right,
                         g.nbhs, g.conn)]
        a = self._arrays
        self._grid = _lib.Grid(self.n, *[_ptr(v) for v in a], self.n, g.shapes)
        h = C.c_void_p()
        st = self.lib.mfcfd_create(C.byref(self._grid), C.byref(self.params), C.byref(h))
        _lib.check(st, None, "mfcfd_create")
        self.h = h
        self.halted = False

    def close(self):
        if getattr(self, "h", None):
            self.lib.mfcfd_destroy(self.h)
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

    # state -------------------------------------------------------------
    def set_state(self, prim: np.ndarray) -> None:
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        if prim.shape != (self.n, 4):
            raise ValueError(f"prim must be ({self.n}, 4)")
        _lib.check(self.lib.mfcfd_set_state(self.h, _dptr(prim)), self.h, "mfcfd_set_state")

    def get_state(self) -> np.ndarray:
        out = np.empty((self.n, 4))
        _lib.check(self.lib.mfcfd_get_state(self.h, _dptr(out)), self.h, "mfcfd_get_state")
        return out

    prim = get_state

    # loop ----------------------------------------------------------------
    def run(self, n_iters: int, it_first: int | None = None) -> np.ndarray:
        """Runs ``n_iters`` iterations; returns the residue of each one done."""
        if it_first is None:
            it_first = (self.it or 0) + 1
        res = np.zeros(max(n_iters, 1))
        done = C.c_int(0)
        st = self.lib.mfcfd_run(self.h, int(it_first), int(n_iters), _dptr(res), C.byref(done))
        self.it = it_first + done.value - 1
        if st == _lib.MFCFD_ERR_NONFINITE:
            self.halted = True
        else:
            _lib.check(st, self.h, "mfcfd_run")
        return res[:done.value].copy()

    def forces(self):
        """(Cl, Cd, Cm) per shape and cp per shape point (grid order)."""
        s = self.grid.shapes
        cl, cd, cm = np.zeros(s), np.zeros(s), np.zeros(s)
        cp = np.zeros(int((self.grid.flag_2 > 0).sum()))
        _lib.check(self.lib.mfcfd_forces(self.h, _dptr(cl), _dptr(cd), _dptr(cm), _dptr(cp)),
                   self.h, "mfcfd_forces")
        return cl, cd, cm, cp

    def adjoint(self, n_iters: int, objective: str = "cd", ckpt_bytes: int = 2 << 30):
        """dJ/dx, dJ/dy per point for J = Cl or Cd after ``n_iters`` iterations
        from the current state (reverse mode, binomial checkpointing).
        Returns (J, dJdx, dJdy, forward iterations run)."""
        dx, dy = np.zeros(self.n), np.zeros(self.n)
        J = C.c_double(0.0)
        nf = C.c_int(0)
        obj = _lib.OBJECTIVES[objective.lower()]
        _lib.check(self.lib.mfcfd_adjoint(self.h, obj, int(n_iters), int(ckpt_bytes),
                                          C.byref(J), _dptr(dx), _dptr(dy), C.byref(nf)),
                   self.h, "mfcfd_adjoint")
        self.it = (self.it or 0) + n_iters
        return J.value, dx, dy, nf.value

    def objective(self, objective: str = "cd") -> float:
        """J of the current state: "cl", "cd" (summed over shapes), "entropy",
        "enstrophy" or "stagnation" (the reference's objective routines)."""
        J = C.c_double(0.0)
        _lib.check(self.lib.mfcfd_objective(self.h, _lib.OBJECTIVES[objective.lower()],
                                            C.byref(J)), self.h, "mfcfd_objective")
        return J.value

    def output_fields(self):
        """(mach, entropy, sensor, total entropy) of the current state: the
        CUDA tree's output.dat columns (post_processing.F90:7-36,
        compute_entropy.F90:10-30, adaptation_sensors.F90:7-101)."""
        mach, ent, sen = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        tot = C.c_double(0.0)
        _lib.check(self.lib.mfcfd_output_fields(self.h, _dptr(mach), _dptr(ent), _dptr(sen),
                                                C.byref(tot)), self.h, "mfcfd_output_fields")
        return mach, ent, sen, tot.value

    def tangent(self, n_iters: int, dx=None, dy=None, objective: str = "cd"):
        """Forward-mode derivative: (J, dJ/de) after ``n_iters`` iterations
        from the current state with the grid moved along (dx, dy) per point
        (forward mode; the state is left unchanged)."""
        def arr(a):
            return None if a is None else _dptr(np.ascontiguousarray(a, dtype=np.float64))
        keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (dx, dy) if a is not None]
        J, dJ = C.c_double(0.0), C.c_double(0.0)
        obj = _lib.OBJECTIVES[objective.lower()]
        pdx = _dptr(keep[0]) if dx is not None else None
        pdy = _dptr(keep[-1]) if dy is not None else None
        _lib.check(self.lib.mfcfd_tangent(self.h, obj, int(n_iters), pdx, pdy, C.byref(J),
                                          C.byref(dJ)), self.h, "mfcfd_tangent")
        return J.value, dJ.value

    # diagnostics -----------------------------------------------------------
    def keep_diagnostics(self, on: bool = True) -> None:
        _lib.check(self.lib.mfcfd_keep_diagnostics(self.h, 1 if on else 0), self.h,
                   "mfcfd_keep_diagnostics")

    _WIDTH = {"q": 4, "dq": 8, "qm": 8, "delta": 1, "flux_res": 4, "nx": 1, "ny": 1}

    def get_array(self, name: str) -> np.ndarray:
        w = self._WIDTH[name]
        out = np.empty(self.n * w)
        _lib.check(self.lib.mfcfd_get_array(self.h, name.encode(), _dptr(out)), self.h,
                   f"mfcfd_get_array({name})")
        return out.reshape(self.n, w) if w > 1 else out

    def profile_iteration(self) -> dict:
        """Runs the next iteration with CUDA events around every kernel; mean
        ms per launch of each kernel kind and of the whole iteration."""
        it = (self.it or 0) + 1
        ms = np.zeros(5)
        _lib.check(self.lib.mfcfd_profile_iteration(self.h, it, _dptr(ms)), self.h,
                   "mfcfd_profile_iteration")
        self.it = it
        return dict(grad=ms[0], inner=ms[1], flux=ms[2], residual=ms[3], iteration=ms[4])

    def set_stream(self, stream_ptr: int | None) -> None:
        _lib.check(self.lib.mfcfd_set_stream(self.h, C.c_void_p(stream_ptr or 0)), self.h,
                   "mfcfd_set_stream")

    def launch_count(self) -> int:
        return int(self.lib.mfcfd_launch_count(self.h))

    def info(self):
        v = [C.c_int() for _ in range(4)]
        _lib.check(self.lib.mfcfd_info(self.h, *[C.byref(x) for x in v]), self.h, "mfcfd_info")
        return tuple(x.value for x in v)


def adjoint_many(solvers, n_iters: int, objective: str = "cd", ckpt_bytes: int = 2 << 30):
    """``Solver.adjoint`` of many independent solvers in one call
    (``mfcfd_adjoint_many``): their reverse sweeps run side by side, each on
    its solver's own stream.  Returns one (J, dJdx, dJdy, forward iterations)
    per solver, each equal to what ``Solver.adjoint`` gives on it."""
    solvers = list(solvers)
    n = len(solvers)
    if n == 0:
        return []
    lib = solvers[0].lib
    handles = (C.c_void_p * n)(*[s.h for s in solvers])
    dx = [np.zeros(s.n) for s in solvers]
    dy = [np.zeros(s.n) for s in solvers]
    px = (C.POINTER(C.c_double) * n)(*[_dptr(a) for a in dx])
    py = (C.POINTER(C.c_double) * n)(*[_dptr(a) for a in dy])
    J = np.zeros(n)
    nf = np.zeros(n, dtype=np.int32)
    st = np.zeros(n, dtype=np.int32)
    ip = C.POINTER(C.c_int)
    rc = lib.mfcfd_adjoint_many(n, handles, _lib.OBJECTIVES[objective.lower()], int(n_iters),
                                int(ckpt_bytes), _dptr(J), px, py, nf.ctypes.data_as(ip),
                                st.ctypes.data_as(ip))
    if rc != _lib.MFCFD_OK:
        bad = [k for k in range(n) if st[k] != _lib.MFCFD_OK] or [0]
        _lib.check(rc, solvers[bad[0]].h, f"mfcfd_adjoint_many (solver {bad[0]})")
    for s in solvers:
        s.it = (s.it or 0) + n_iters
    return [(float(J[k]), dx[k], dy[k], int(nf[k])) for k in range(n)]
