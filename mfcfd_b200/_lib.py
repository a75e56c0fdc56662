"""ctypes binding of the C ABI declared in include/mfcfd_b200.h.

The product path has no fallback: if libmfcfd_b200.so is missing and cannot
be built, or the CUDA device is absent, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

MFCFD_OK = 0
MFCFD_ERR_ARG = -1
MFCFD_ERR_CUDA = -2
MFCFD_ERR_NONFINITE = -3
MFCFD_ERR_TIMEOUT = -4
MFCFD_ERR_OOM = -5
MFCFD_ERR_GRID = -6
MFCFD_ERR_NODEV = -7
MFCFD_ERR_STATE = -8
MFCFD_FP64 = 0
MFCFD_FP32_MIXED = 1
MFCFD_ORDER_KIND = 0
MFCFD_ORDER_RCM = 1

# every symbol include/mfcfd_b200.h declares
EXPORTS = ("mfcfd_default_params", "mfcfd_create", "mfcfd_destroy", "mfcfd_set_state",
           "mfcfd_get_state", "mfcfd_run", "mfcfd_forces", "mfcfd_set_stream",
           "mfcfd_get_array", "mfcfd_keep_diagnostics", "mfcfd_info", "mfcfd_strerror",
           "mfcfd_last_error", "mfcfd_launch_count", "mfcfd_profile_iteration",
           "mfcfd_measure_fp64_peak", "mfcfd_create_part", "mfcfd_part_phase",
           "mfcfd_part_rows", "mfcfd_part_index",
           "mfcfd_run_noalloc", "mfcfd_adjoint", "mfcfd_adjoint_many", "mfcfd_tangent",
           "mfcfd_output_fields",
           "mfcfd_objective",
           "mfcfd_batch_create", "mfcfd_batch_destroy",
           "mfcfd_batch_set_stream", "mfcfd_batch_set_state", "mfcfd_batch_get_state",
           "mfcfd_batch_run", "mfcfd_batch_forces", "mfcfd_batch_tune", "mfcfd_batch_set_launch",
           "mfcfd_batch_info", "mfcfd_batch_last_error", "mfcfd_batch_launch_count")
MFCFD_BATCH_MAX = 256
MFCFD_ADJOINT_MANY_MAX = 256
OBJECTIVES = {"cl": 0, "cd": 1, "entropy": 2, "enstrophy": 3, "stagnation": 4}
BATCH_STATES = {0: "running", 1: "converged", 2: "max_iters", 3: "nonfinite"}
MFCFD_NOALLOC_MAX_ITERS = 65536
PHASE_BEGIN, PHASE_GRAD, PHASE_INNER, PHASE_FLUX, PHASE_GHOSTS, PHASE_END = range(6)


class Grid(C.Structure):
    _fields_ = [("n", C.c_int), ("x", C.c_void_p), ("y", C.c_void_p), ("nx", C.c_void_p),
                ("ny", C.c_void_p), ("min_dist", C.c_void_p), ("flag_1", C.c_void_p),
                ("flag_2", C.c_void_p), ("left", C.c_void_p), ("right", C.c_void_p),
                ("nbhs", C.c_void_p), ("conn", C.c_void_p), ("ld_conn", C.c_int),
                ("shapes", C.c_int)]


class Params(C.Structure):
    _fields_ = [("cfl", C.c_double), ("power", C.c_double), ("vl_const", C.c_double),
                ("mach", C.c_double), ("aoa", C.c_double), ("rks", C.c_int),
                ("euler", C.c_double), ("inner_iterations", C.c_int),
                ("interior_points_normal_flag", C.c_int), ("format", C.c_int),
                ("restart", C.c_int), ("res_old", C.c_double), ("precision", C.c_int),
                ("ordering", C.c_int)]


_LIB = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True) -> C.CDLL:
    """Loads libmfcfd_b200.so (building it in-tree first if it is absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.LIB
    if not os.path.exists(path) or (build_if_missing and not _build.up_to_date()):
        if not build_if_missing:
            raise RuntimeError(f"{path} is missing")
        _build.build()
    lib = C.CDLL(path)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    I = C.POINTER(C.c_int)
    lib.mfcfd_default_params.argtypes = [C.POINTER(Params)]
    lib.mfcfd_create.argtypes = [C.POINTER(Grid), C.POINTER(Params), C.POINTER(P)]
    lib.mfcfd_destroy.argtypes = [P]
    lib.mfcfd_set_state.argtypes = [P, D]
    lib.mfcfd_get_state.argtypes = [P, D]
    lib.mfcfd_run.argtypes = [P, C.c_int, C.c_int, D, I]
    lib.mfcfd_forces.argtypes = [P, D, D, D, D]
    lib.mfcfd_set_stream.argtypes = [P, P]
    lib.mfcfd_get_array.argtypes = [P, C.c_char_p, D]
    lib.mfcfd_keep_diagnostics.argtypes = [P, C.c_int]
    lib.mfcfd_info.argtypes = [P, I, I, I, I]
    lib.mfcfd_strerror.argtypes = [C.c_int]
    lib.mfcfd_strerror.restype = C.c_char_p
    lib.mfcfd_last_error.argtypes = [P]
    lib.mfcfd_last_error.restype = C.c_char_p
    lib.mfcfd_launch_count.argtypes = [P]
    lib.mfcfd_launch_count.restype = C.c_longlong
    lib.mfcfd_profile_iteration.argtypes = [P, C.c_int, D]
    lib.mfcfd_measure_fp64_peak.argtypes = [D]
    lib.mfcfd_create_part.argtypes = [C.POINTER(Grid), C.POINTER(Params), C.c_int, C.c_int,
                                      C.POINTER(P)]
    lib.mfcfd_part_phase.argtypes = [P, C.c_int, C.c_int, C.c_int, D]
    lib.mfcfd_part_rows.argtypes = [P, C.c_char_p, C.POINTER(C.c_void_p), I]
    lib.mfcfd_part_index.argtypes = [P, I]
    lib.mfcfd_run_noalloc.argtypes = [P, C.c_int, C.c_int, D, I]
    lib.mfcfd_adjoint.argtypes = [P, C.c_int, C.c_int, C.c_size_t, D, D, D, I]
    lib.mfcfd_adjoint_many.argtypes = [C.c_int, C.POINTER(P), C.c_int, C.c_int, C.c_size_t, D,
                                       C.POINTER(D), C.POINTER(D), I, I]
    lib.mfcfd_tangent.argtypes = [P, C.c_int, C.c_int, D, D, D, D]
    lib.mfcfd_output_fields.argtypes = [P, D, D, D, D]
    lib.mfcfd_objective.argtypes = [P, C.c_int, D]
    lib.mfcfd_batch_create.argtypes = [C.c_int, C.POINTER(C.POINTER(Grid)), C.POINTER(Params),
                                       C.POINTER(P)]
    lib.mfcfd_batch_destroy.argtypes = [P]
    lib.mfcfd_batch_set_stream.argtypes = [P, P]
    lib.mfcfd_batch_set_state.argtypes = [P, C.c_int, D]
    lib.mfcfd_batch_get_state.argtypes = [P, C.c_int, D]
    lib.mfcfd_batch_run.argtypes = [P, C.c_double, C.c_int, I, I, D]
    lib.mfcfd_batch_forces.argtypes = [P, C.c_int, D, D, D, D]
    lib.mfcfd_batch_tune.argtypes = [P, C.c_int, D]
    lib.mfcfd_batch_set_launch.argtypes = [P, C.c_int, C.c_int, C.c_int]
    lib.mfcfd_batch_info.argtypes = [P, I, C.POINTER(C.c_longlong), I, I, I]
    lib.mfcfd_batch_last_error.argtypes = [P]
    lib.mfcfd_batch_last_error.restype = C.c_char_p
    lib.mfcfd_batch_launch_count.argtypes = [P]
    lib.mfcfd_batch_launch_count.restype = C.c_longlong
    for name in EXPORTS:
        if name not in ("mfcfd_strerror", "mfcfd_last_error", "mfcfd_launch_count",
                        "mfcfd_batch_last_error", "mfcfd_batch_launch_count"):
            getattr(lib, name).restype = C.c_int
    _LIB = lib
    return lib


class MfcfdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


def check(status: int, handle=None, what: str = "") -> None:
    if status == MFCFD_OK:
        return
    lib = load()
    detail = lib.mfcfd_last_error(handle).decode(errors="replace")
    text = lib.mfcfd_strerror(status).decode()
    raise MfcfdError(status, f"{what}: {text}" + (f": {detail}" if detail else ""))
