"""CPU oracle for the LSKUM pseudo-time loop -- TEST INFRASTRUCTURE ONLY.

A ctypes wrapper over ``oracle/_build/liblskum_oracle.so``, the plain-C FP64
restatement of the reference's src_mpi_primal routines.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use it, as the
checker or the timed CPU baseline; the product (``mfcfd_b200``) never does.

Parity status: UNPINNED (the reference has no tests, golden vectors or grids
for this path and its toolchain is absent, so the restatement is checked only
against its own committed fixtures and analytic properties).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_LIBS: dict = {}


class OrcParams(C.Structure):
    _fields_ = [("cfl", C.c_double), ("power", C.c_double), ("vl_const", C.c_double),
                ("mach", C.c_double), ("aoa", C.c_double), ("rks", C.c_int),
                ("euler", C.c_double), ("inner_iterations", C.c_int),
                ("interior_points_normal_flag", C.c_int), ("format", C.c_int),
                ("shapes", C.c_int), ("restart", C.c_int), ("res_old", C.c_double)]


def build() -> None:
    """Compile both oracle variants (make, system gcc)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(variant: str = "") -> C.CDLL:
    name = f"liblskum_oracle{variant}.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(_BUILD, name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P, D, I = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    lib.orc_create.restype = P
    lib.orc_create.argtypes = [C.c_int, D, D, D, D, D, I, I, I, I, I, I, C.c_int,
                               C.POINTER(OrcParams)]
    lib.orc_create_part.restype = P
    lib.orc_create_part.argtypes = [C.c_int, C.c_int, C.c_int, D, D, D, D, D, I, I, I, I, I,
                                    I, C.c_int, C.POINTER(OrcParams)]
    lib.orc_destroy.argtypes = [P]
    lib.orc_set.argtypes = [P, C.c_char_p, D]
    lib.orc_set.restype = C.c_int
    for fn in ("orc_init_freestream", "orc_func_delta", "orc_eval_q_variables",
               "orc_eval_q_derivatives", "orc_eval_q_inner_loop",
               "orc_eval_update_innerloop", "orc_cal_flux_residual", "orc_save_prim_old"):
        getattr(lib, fn).argtypes = [P]
    lib.orc_state_update.argtypes = [P, C.c_int]
    lib.orc_set_prim.argtypes = [P, D]
    lib.orc_get_prim.argtypes = [P, D]
    lib.orc_run.argtypes = [P, C.c_int, C.c_int, D, I]
    lib.orc_run.restype = C.c_int
    lib.orc_forces.argtypes = [P, D, D, D, D]
    lib.orc_get.argtypes = [P, C.c_char_p, D]
    lib.orc_get.restype = C.c_int
    lib.orc_get_split_counts.argtypes = [P, I]
    lib.orc_sum_res_sqr.argtypes = [P]
    lib.orc_output_fields.argtypes = [P, D, D, D]
    lib.orc_output_fields.restype = C.c_double
    lib.orc_objective.argtypes = [P, C.c_int]
    lib.orc_objective.restype = C.c_double
    lib.orc_sum_res_sqr.restype = C.c_double
    lib.orc_num_threads.restype = C.c_int
    _LIBS[name] = lib
    return lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


_SIZES = {"prim": 4, "prim_old": 4, "q": 4, "dq": 8, "qm": 8, "flux_res": 4,
          "delta": 1, "nx": 1, "ny": 1, "temp": 12}


class Oracle:
    """One oracle instance over a grid (reference semantics, original order)."""

    def __init__(self, grid, cfl=0.2, power=0.0, vl_const=5.0, mach=0.63, aoa=2.0,
                 tscheme="ssprk43", inner_iterations=0, interior_points_normal_flag=0,
                 format=1, restart=0, res_old=0.0, variant="", n_local=None, plen=None):
        """n_local / plen: one rank's part of a partitioned grid -- points
        beyond n_local are ghosts (refreshed by the caller with ``put``), and
        the residual norm divides by plen, the global point count."""
        self.lib = _lib(variant)
        self.grid = grid
        self.n = grid.n
        rks, euler = (4, 1.0) if tscheme == "ssprk43" else (1, 2.0)
        self.params = OrcParams(cfl, power, vl_const, mach, aoa, rks, euler,
                                inner_iterations, interior_points_normal_flag, format,
                                grid.shapes, restart, res_old)
        g = grid
        self._keep = [np.ascontiguousarray(a) for a in
                      (g.x, g.y, g.nx, g.ny, g.min_dist, g.flag_1, g.flag_2, g.left,
                       g.right, g.nbhs, g.conn)]
        k = self._keep
        self.n_local = self.n if n_local is None else int(n_local)
        self.h = self.lib.orc_create_part(self.n, self.n_local,
                                          self.n if plen is None else int(plen),
                                          _d(k[0]), _d(k[1]), _d(k[2]), _d(k[3]),
                                          _d(k[4]), _i(k[5]), _i(k[6]), _i(k[7]), _i(k[8]),
                                          _i(k[9]), _i(k[10]), self.n, C.byref(self.params))

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    __del__ = close

    def set_prim(self, prim):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        assert prim.shape == (self.n, 4)
        self.lib.orc_set_prim(self.h, _d(prim))

    def prim(self):
        out = np.empty((self.n, 4))
        self.lib.orc_get_prim(self.h, _d(out))
        return out

    def get(self, name):
        out = np.empty(self.n * _SIZES[name])
        if self.lib.orc_get(self.h, name.encode(), _d(out)) != 0:
            raise KeyError(name)
        return out.reshape(self.n, -1) if _SIZES[name] > 1 else out

    def put(self, name, values):
        """Copies a whole array in ("prim" (n,4), "dq" / "qm" (n,8))."""
        a = np.ascontiguousarray(values, dtype=np.float64)
        if self.lib.orc_set(self.h, name.encode(), _d(a)) != 0:
            raise KeyError(name)

    def split_counts(self):
        out = np.empty((self.n, 4), dtype=np.int32)
        self.lib.orc_get_split_counts(self.h, _i(out))
        return out

    def run(self, n_iters, it_first=1):
        res = np.zeros(max(n_iters, 1))
        done = C.c_int(0)
        self.lib.orc_run(self.h, it_first, n_iters, _d(res), C.byref(done))
        return res[:done.value]

    def forces(self):
        s = self.grid.shapes
        cl, cd, cm = np.zeros(s), np.zeros(s), np.zeros(s)
        cp = np.zeros(int((self.grid.flag_2 > 0).sum()))
        self.lib.orc_forces(self.h, _d(cl), _d(cd), _d(cm), _d(cp))
        return cl, cd, cm, cp

    # stage-level access
    def output_fields(self):
        """(mach, entropy, sensor, total entropy) of the current state: the CUDA
        tree's post-processing fields (src_cuda/post_processing.F90:7-36,
        compute_entropy.F90:10-30, adaptation_sensors.F90:7-101)."""
        n = self.grid.n
        mach, ent, sen = np.zeros(n), np.zeros(n), np.zeros(n)
        tot = self.lib.orc_output_fields(self.h, _d(mach), _d(ent), _d(sen))
        return mach, ent, sen, tot

    def objective(self, kind: str):
        """J of the current state: "cl"/"cd" (summed over shapes) or a
        secondary objective "entropy", "enstrophy", "stagnation"."""
        if kind in ("cl", "cd"):
            cl, cd, _, _ = self.forces()
            return float((cd if kind == "cd" else cl).sum())
        k = {"entropy": 2, "enstrophy": 3, "stagnation": 4}[kind]
        return float(self.lib.orc_objective(self.h, k))

    def func_delta(self): self.lib.orc_func_delta(self.h)
    def q_variables(self): self.lib.orc_eval_q_variables(self.h)
    def q_derivatives(self): self.lib.orc_eval_q_derivatives(self.h)
    def q_inner_loop(self): self.lib.orc_eval_q_inner_loop(self.h)
    def update_innerloop(self): self.lib.orc_eval_update_innerloop(self.h)
    def flux_residual(self): self.lib.orc_cal_flux_residual(self.h)
    def state_update(self, rk): self.lib.orc_state_update(self.h, rk)
    def save_prim_old(self): self.lib.orc_save_prim_old(self.h)
    def sum_res_sqr(self): return self.lib.orc_sum_res_sqr(self.h)


def num_threads(variant: str = "") -> int:
    return int(_lib(variant).orc_num_threads())
