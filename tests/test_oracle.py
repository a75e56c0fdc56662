"""CPU tests of the oracle: golden fixtures, reference properties, invariants.

The reference has no tests or golden data for this path (parity unpinned);
these pin the restatement against its committed fixtures, the FMA-contracted
build, and properties the reference's algorithm has by construction.
"""
import os

import numpy as np
import pytest

import oracle
from mfcfd_b200.grid import naca_ogrid
from tests.golden.make_golden import CASES, case_grid
from tests.helpers import max_rel, max_scaled

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden(name):
    gk, flow, iters = CASES[name]
    ref = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    g = case_grid(name)
    o = oracle.Oracle(g, **flow)
    r1 = o.run(1)
    for a in ("prim", "q", "dq", "qm", "flux_res", "delta"):
        assert max_scaled(o.get(a), ref[f"it1_{a}"]) < 1e-13, a
    r = o.run(iters - 1, it_first=2)
    assert np.allclose(np.concatenate([r1, r]), ref["residue"], rtol=0, atol=1e-12)
    assert max_rel(o.prim(), ref["prim"]) < 1e-12
    cl, cd, cm, cp = o.forces()
    assert np.allclose([cl[0], cd[0], cm[0]], [ref["cl"][0], ref["cd"][0], ref["cm"][0]],
                       rtol=0, atol=1e-12)
    assert max_scaled(cp[:, None], ref["cp"][:, None]) < 1e-12


def test_fma_build_agrees():
    """The FMA-contracted build (what gfortran -O3 -march=native does) stays
    within rounding of the parity build: bounds the rounding sensitivity."""
    g = case_grid("plain")
    _, flow, _ = CASES["plain"]
    a = oracle.Oracle(g, **flow)
    b = oracle.Oracle(g, variant="_fma", **flow)
    ra, rb = a.run(12), b.run(12)
    assert max_rel(a.prim(), b.prim()) < 1e-11
    assert np.allclose(ra, rb, rtol=0, atol=1e-10)


def test_freestream_preserved_in_interior():
    """A uniform state gives dq = 0 and zero flux residual everywhere; only
    the wall condition (U(3) = 0) changes the state in the first stage."""
    g = naca_ogrid(32, 12, seed=3, first_spacing=5e-3)
    o = oracle.Oracle(g, cfl=0.2, vl_const=5.0, mach=0.5, aoa=3.0)
    o.save_prim_old()
    o.func_delta()
    o.q_variables()
    o.q_derivatives()
    assert np.all(o.get("dq") == 0.0)
    o.flux_residual()
    assert np.all(o.get("flux_res") == 0.0)
    p0 = o.prim()
    o.state_update(1)
    p1 = o.prim()
    interior = g.flag_1 == 1
    # prim -> conserved -> prim round trip: unchanged up to rounding
    assert max_rel(p1[interior], p0[interior]) < 2e-15
    wall = g.flag_1 == 0
    nx, ny = o.get("nx")[wall], o.get("ny")[wall]
    un = p1[wall, 1] * nx + p1[wall, 2] * ny
    assert np.max(np.abs(un)) < 1e-15


def test_mirror_symmetry_at_zero_incidence():
    """aoa = 0 on a jitter-free symmetric grid: the solution is symmetric
    about the chord line (rho, u1, p even; u2 odd) -- checks every sign in the
    split fluxes, the y split and the wall/outer treatment."""
    ni, nj = 48, 16
    g = naca_ogrid(ni, nj, jitter=0.0, first_spacing=5e-3)
    o = oracle.Oracle(g, cfl=0.2, vl_const=5.0, mach=0.6, aoa=0.0)
    o.run(20)
    p = o.prim().reshape(nj, ni, 4)
    mirror = p[:, (-np.arange(ni)) % ni, :]
    assert np.max(np.abs(p[..., 0] - mirror[..., 0])) < 1e-9
    assert np.max(np.abs(p[..., 1] - mirror[..., 1])) < 1e-9
    assert np.max(np.abs(p[..., 2] + mirror[..., 2])) < 1e-9
    assert np.max(np.abs(p[..., 3] - mirror[..., 3])) < 1e-9
    cl, cd, cm, _ = o.forces()
    assert abs(cl[0]) < 1e-9


def test_nan_exit_stops_the_loop():
    """q_lskum.F90:71: the loop ends after the first NaN residue."""
    g = naca_ogrid(32, 12, seed=5, first_spacing=5e-3)
    o = oracle.Oracle(g, cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0)
    p = o.prim()
    p[100, 3] = -1.0  # negative pressure: log of a negative beta
    o.set_prim(p)
    r = o.run(10)
    assert len(r) < 10 and np.isnan(r[-1])


def test_residue_is_zero_for_first_two_iterations():
    g = naca_ogrid(32, 12, seed=5, first_spacing=5e-3)
    o = oracle.Oracle(g, cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0)
    r = o.run(4)
    assert r[0] == 0.0 and r[1] == 0.0 and r[2] != 0.0
    o2 = oracle.Oracle(g, cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0, restart=1, res_old=1e-3)
    r2 = o2.run(2)
    assert r2[0] != 0.0


def test_oracle_thread_count_independent(monkeypatch):
    """Per-point loops write only their own point: results do not depend on
    the OpenMP thread count (the serial reductions keep reference order)."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import numpy as np, oracle;"
            "from tests.golden.make_golden import CASES, case_grid;"
            "g = case_grid('plain'); f = CASES['plain'][1];"
            "o = oracle.Oracle(g, **f); r = o.run(5);"
            "sys.stdout.write(repr(float(np.sum(o.prim()))) + repr(r.tolist()))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = []
    for t in ("1", "3"):
        env = dict(os.environ, OMP_NUM_THREADS=t)
        outs.append(subprocess.run([sys.executable, "-c", code % root], env=env, cwd=root,
                                   capture_output=True, text=True, check=True).stdout)
    assert outs[0] == outs[1]
