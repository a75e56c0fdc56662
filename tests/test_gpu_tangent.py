"""Forward-mode derivative (mfcfd_tangent) against the reverse mode and
finite differences.

The reference differentiates its loop in both modes with Tapenade
(src_mpi_forward/sensitivity_files/q_lskum_d.F90:28-89 seeds pointd%x(1) = 1;
src_mpi_adjoint for the reverse).  The classic check of a hand-written
adjoint is the dot-product test: for any direction d, the tangent dJ/de
equals <dJ/d(x, y), d> from the adjoint.  Tolerances: 1e-9 relative for the
dot product (both are exact derivatives up to rounding), 1e-6 relative for
central differences with h = 1e-7.
"""
import copy

import numpy as np
import pytest

from mfcfd_b200 import _lib
from mfcfd_b200.grid import naca_ogrid
from mfcfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _flow(**kw):
    f = dict(cfl=0.2, vl_const=5.0, mach=0.6, aoa=2.0)
    f.update(kw)
    return f


@pytest.mark.parametrize("obj,inner,tscheme,n", [("cd", 0, "ssprk43", 3), ("cl", 1, "ssprk43", 2),
                                                 ("cd", 0, "first", 4)])
def test_dot_product_with_the_adjoint(gpu, obj, inner, tscheme, n):
    g = naca_ogrid(32, 12, seed=5, first_spacing=5e-3)
    f = _flow(inner_iterations=inner, tscheme=tscheme)
    rng = np.random.default_rng(11)
    dx, dy = rng.standard_normal(g.n), rng.standard_normal(g.n)
    with Solver(g, **f) as s:
        s.run(2)
        p0 = s.get_state()
        Jt, dJt = s.tangent(n, dx, dy, objective=obj)
        assert np.array_equal(s.get_state(), p0)  # the tangent leaves the state alone
        Ja, gx, gy, _ = s.adjoint(n, obj)
    dot = float(gx @ dx + gy @ dy)
    assert abs(Jt - Ja) <= 1e-12 * abs(Ja)
    assert abs(dJt - dot) <= 1e-9 * max(abs(dot), np.abs(gx).sum() + np.abs(gy).sum()), (dJt, dot)


def test_tangent_matches_central_differences(gpu):
    # An odd ni: the even-ni grids are exact mirror images, whose aligned
    # points tie at dels/deln = 0 and sit in both split lists; a random
    # perturbation breaks the ties, a jump in J that no derivative sees.
    g = naca_ogrid(31, 12, seed=6, first_spacing=5e-3)
    f = _flow(inner_iterations=1)
    n, h = 3, 1e-7
    rng = np.random.default_rng(12)
    dx, dy = rng.standard_normal(g.n), rng.standard_normal(g.n)
    with Solver(g, **f) as s:
        _, dJt = s.tangent(n, dx, dy)
    J = []
    for sgn in (1.0, -1.0):
        gs = copy.deepcopy(g)
        gs.x = g.x + sgn * h * dx
        gs.y = g.y + sgn * h * dy
        with Solver(gs, **f) as s:
            s.run(n)
            J.append(float(s.forces()[1].sum()))
    fd = (J[0] - J[1]) / (2 * h)
    assert abs(dJt - fd) <= 1e-6 * abs(fd) + 1e-9, (dJt, fd)


def test_reference_seed_is_one_gradient_entry(gpu):
    # Q_LSKUM_D's seed: d/dx of point 1 only
    g = naca_ogrid(24, 10, seed=8, first_spacing=5e-3)
    f = _flow()
    dx = np.zeros(g.n)
    dx[0] = 1.0
    with Solver(g, **f) as s:
        _, dJt = s.tangent(3, dx, None)
        _, gx, _, _ = s.adjoint(3, "cd")
    assert abs(dJt - gx[0]) <= 1e-9 * max(abs(gx[0]), 1e-12) + 1e-15


def test_tangent_rejects_unsupported_handles(gpu):
    g = naca_ogrid(24, 10, seed=8, first_spacing=5e-3)
    for kw in (dict(precision="fp32_mixed"), dict(power=-2.0)):
        with Solver(g, **_flow(**kw)) as s:
            with pytest.raises(_lib.MfcfdError):
                s.tangent(1)
