"""Secondary objectives (MFCFD_OBJ_ENTROPY / ENSTROPHY / STAGNATION): the
value against the oracle, and their derivatives three ways -- the reverse
mode against central differences of the GPU primal, and the forward mode
against the reverse mode (dot-product test).  The state the derivative
starts from is 20 iterations in (held fixed), off the freestream, where the
entropy term |t| would sit on its kink t = 0."""
import copy

import numpy as np
import pytest

import oracle
from mfcfd_b200.grid import naca_ogrid
from mfcfd_b200.solver import Solver

pytestmark = pytest.mark.gpu

SECONDARY = ["entropy", "enstrophy", "stagnation"]
FLOW = dict(cfl=0.2, vl_const=5.0, mach=0.65, aoa=1.5)


def _start(g):
    with Solver(g, **FLOW) as s:
        s.run(20)
        return s.get_state()


def test_objective_values_match_the_oracle(gpu):
    g = naca_ogrid(40, 14, seed=3, first_spacing=5e-3)
    with Solver(g, **FLOW) as s:
        s.run(10)
        prim = s.get_state()
        J = {k: s.objective(k) for k in ["cl", "cd"] + SECONDARY}
    o = oracle.Oracle(g, **FLOW)
    o.set_prim(prim)
    for k, v in J.items():
        ref = o.objective(k)
        assert abs(v - ref) <= 1e-12 * abs(ref), (k, v, ref)
    o.close()


@pytest.mark.parametrize("obj", SECONDARY)
def test_secondary_adjoint_matches_finite_differences(gpu, obj):
    g = naca_ogrid(31, 12, seed=5, first_spacing=5e-3)
    prim0 = _start(g)
    n, h = 3, 1e-7
    with Solver(g, **FLOW) as s:
        s.set_state(prim0)
        J, dx, dy, _ = s.adjoint(n, obj)

    def Jof(gg):
        with Solver(gg, **FLOW) as s:
            s.set_state(prim0)
            s.run(n)
            return s.objective(obj)

    assert abs(J - Jof(g)) <= 1e-12 * abs(J)
    rng = np.random.default_rng(3)
    worst = 0.0
    fds = []
    for p in rng.choice(np.arange(g.n), size=8, replace=False):
        for arr, grad in (("x", dx), ("y", dy)):
            gp, gm = copy.deepcopy(g), copy.deepcopy(g)
            getattr(gp, arr)[p] += h
            getattr(gm, arr)[p] -= h
            fd = (Jof(gp) - Jof(gm)) / (2 * h)
            fds.append(fd)
            worst = max(worst, abs(grad[p] - fd))
    assert worst <= 1e-6 * max(np.abs(fds).max(), 1e-12) + 1e-9 * abs(J), worst


@pytest.mark.parametrize("obj", SECONDARY)
def test_secondary_dot_product(gpu, obj):
    g = naca_ogrid(32, 12, seed=6, first_spacing=5e-3)
    prim0 = _start(g)
    rng = np.random.default_rng(7)
    ddx, ddy = rng.standard_normal(g.n), rng.standard_normal(g.n)
    with Solver(g, **FLOW) as s:
        s.set_state(prim0)
        Jt, dJt = s.tangent(3, ddx, ddy, objective=obj)
        Ja, gx, gy, _ = s.adjoint(3, obj)
    dot = float(gx @ ddx + gy @ ddy)
    assert abs(Jt - Ja) <= 1e-12 * abs(Ja)
    assert abs(dJt - dot) <= 1e-9 * max(abs(dot), np.abs(gx).sum() + np.abs(gy).sum()), (dJt, dot)
