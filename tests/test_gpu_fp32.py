"""FP32-mixed path: against the FP64 path (and so the oracle) on the same grid.

The FP32-mixed path keeps prim/q/dq/qm and the per-neighbour flux work in
FP32, so it cannot match the oracle to FP64 rounding; its error is bounded
here against the FP64 path after 200 iterations of the 16k configuration:
force coefficients within 1e-5 (the contract), residue history within 1e-3
(log10 units), prim within 1e-4 relative in RMS and 5e-2 at worst (single
points in steep gradients can flip a limiter branch).
"""
import numpy as np
import pytest

from mfcfd_b200.grid import config_flow, config_grid, naca_ogrid
from mfcfd_b200.solver import Solver
from tests.helpers import max_rel

pytestmark = pytest.mark.gpu


def test_fp32_mixed_tracks_fp64(gpu):
    g = config_grid("C1")
    f = config_flow("C1")
    with Solver(g, **f) as a, Solver(g, precision="fp32_mixed", **f) as b:
        ra, rb = a.run(200), b.run(200)
        pa, pb = a.get_state(), b.get_state()
        cla, cda, _, _ = a.forces()
        clb, cdb, _, _ = b.forces()
    rel = np.abs(pb - pa) / np.maximum(np.abs(pa), 1e-3 * np.max(np.abs(pa), axis=0))
    assert np.sqrt(np.mean(rel ** 2)) < 1e-4
    assert rel.max() < 5e-2
    assert np.max(np.abs(ra - rb)) < 1e-3
    assert abs(cla[0] - clb[0]) < 1e-5 and abs(cda[0] - cdb[0]) < 1e-5


def test_fp32_mixed_inner_iterations_and_state_io(gpu):
    g = naca_ogrid(48, 20, seed=51, first_spacing=5e-3)
    f = dict(cfl=0.2, vl_const=5.0, mach=0.8, aoa=1.0, inner_iterations=3)
    with Solver(g, **f) as a, Solver(g, precision="fp32_mixed", **f) as b:
        a.run(10)
        b.run(10)
        assert max_rel(b.get_state(), a.get_state()) < 1e-3
        # state round trip keeps FP32 values exactly
        s = b.get_state()
        b.set_state(s)
        assert np.array_equal(b.get_state(), s)
        dq32, dq64 = b.get_array("dq"), a.get_array("dq")
        scale = np.max(np.abs(dq64), axis=0)
        assert np.max(np.abs(dq32 - dq64) / np.maximum(scale, 1e-12)) < 1e-3


def test_fp32_mixed_fine_trailing_edge(gpu):
    # the C5 wall (2560 cosine-spaced points, first spacing 1e-3, M 0.8):
    # with the trailing-edge stencils repaired every split list is
    # well-posed and FP32-mixed runs as FP64 does
    g = naca_ogrid(2560, 16, seed=5000, first_spacing=1e-3)
    f = dict(config_flow("C5"))
    with Solver(g, **f) as a, Solver(g, precision="fp32_mixed", **f) as b:
        ra, rb = a.run(30), b.run(30)
        assert not a.halted and not b.halted and len(rb) == 30
        cla, cda, _, _ = a.forces()
        clb, cdb, _, _ = b.forces()
    assert np.isfinite(rb).all()
    assert np.max(np.abs(ra - rb)) < 1e-3
    assert abs(cla[0] - clb[0]) < 1e-5 and abs(cda[0] - cdb[0]) < 1e-5
