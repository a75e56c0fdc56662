"""mfcfd_adjoint_many: the adjoints of independent solvers of uneven sizes
in one call equal mfcfd_adjoint on each solver bit for bit (gradients,
objective, forward-iteration count and the final state), under a snapshot
budget that forces recomputation; invalid handle lists are refused before
anything runs."""
import numpy as np
import pytest

from mfcfd_b200._lib import MfcfdError
from mfcfd_b200.grid import batch_instances
from mfcfd_b200.solver import Solver, adjoint_many

pytestmark = pytest.mark.gpu


def _instances():
    grids, flows, _ = batch_instances(4, config=5, n_min=1500, n_max=12000)
    return grids, flows


@pytest.mark.parametrize("objective", ["cd", "cl"])
def test_adjoint_many_matches_single(gpu, objective):
    grids, flows = _instances()
    a = [Solver(g, **f) for g, f in zip(grids, flows)]
    b = [Solver(g, **f) for g, f in zip(grids, flows)]
    try:
        for s in a + b:
            s.run(12)
        iters = 9
        budget = 3 * 32 * max(g.n for g in grids)  # 2-3 snapshots: recomputation
        single = [s.adjoint(iters, objective, ckpt_bytes=budget) for s in a]
        many = adjoint_many(b, iters, objective, ckpt_bytes=budget)
        assert len(many) == len(single)
        for (J1, x1, y1, f1), (J2, x2, y2, f2), sa, sb in zip(single, many, a, b):
            assert J1 == J2 and f1 == f2 and f1 > iters
            assert np.array_equal(x1, x2) and np.array_equal(y1, y2)
            assert np.abs(x1).max() > 0
            assert np.array_equal(sa.get_state(), sb.get_state())
    finally:
        for s in a + b:
            s.close()


def test_adjoint_many_refuses_bad_lists(gpu):
    grids, flows = _instances()
    g, f = grids[0], flows[0]
    with Solver(g, **f) as s, Solver(g, precision="fp32_mixed", **f) as s32, \
            Solver(g, **f) as t:
        s.run(3)
        with pytest.raises(MfcfdError):
            adjoint_many([s, s], 2)
        with pytest.raises(MfcfdError):
            adjoint_many([s, s32], 2)
        assert s.launch_count() > 0
        t.set_stream(None)
        out = adjoint_many([s, t], 2)
        assert len(out) == 2 and np.isfinite(out[0][1]).all()
