"""mfcfd_run_noalloc: the pseudo-time loop for callers that cannot allocate.

A caller whose device memory belongs to its own pool, or a service that
allocates only at start-up, cannot let the library call cudaMalloc while it
runs; mfcfd_run_noalloc keeps its scratch (the residue history) in a fixed
per-device array instead, whose address mfcfd_create looks up.  These checks
call it through the C ABI and compare it with mfcfd_run on an identical
solver, on two calls in a row, and check that the two calls leave the
device's free memory unchanged.  The file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from mfcfd_b200 import _lib
from mfcfd_b200.grid import naca_ogrid
from mfcfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _run_noalloc(s, it_first, n):
    res = np.zeros(max(n, 1))
    done = C.c_int(0)
    st = s.lib.mfcfd_run_noalloc(s.h, it_first, n, res.ctypes.data_as(C.POINTER(C.c_double)),
                                 C.byref(done))
    return st, res[:done.value]


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


def test_run_noalloc_matches_run_on_two_calls(gpu):
    g = naca_ogrid(48, 20, seed=41, first_spacing=5e-3)
    flow = dict(cfl=0.2, vl_const=5.0, mach=0.7, aoa=1.5, inner_iterations=2)
    calls = ((1, 7), (8, 5))  # two calls in a row; the shared array keeps the first's history
    with Solver(g, **flow) as a, Solver(g, **flow) as b:
        ref = []
        for it, n in calls:
            ra = a.run(n, it_first=it)
            ref.append((ra, a.get_state()))
        free0 = _free_bytes()
        for (it, n), (ra, pa) in zip(calls, ref):
            st, rb = _run_noalloc(b, it, n)
            assert st == _lib.MFCFD_OK, b.lib.mfcfd_last_error(b.h)
            # same kernels in the same order on the same inputs: identical bits
            assert len(rb) == len(ra) == n
            assert np.array_equal(rb, ra)
            assert np.array_equal(b.get_state(), pa)
            assert _free_bytes() == free0, "mfcfd_run_noalloc changed the device's free memory"


def test_run_noalloc_rejects_oversized_runs(gpu):
    g = naca_ogrid(24, 10, seed=42, first_spacing=5e-3)
    with Solver(g, cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0) as s:
        st, _ = _run_noalloc(s, 1, _lib.MFCFD_NOALLOC_MAX_ITERS + 1)
        assert st == _lib.MFCFD_ERR_ARG
        assert b"MFCFD_NOALLOC_MAX_ITERS" in s.lib.mfcfd_last_error(s.h)
