"""Batched runs (mfcfd_batch_*) against single-instance runs of the same grids.

Every instance of a batch follows the single-instance loop point by point and
sums its residual partials in the same order, so states, residues, retirement
iterations and forces must be bit-identical to a ``Solver`` of that grid.
"""
import numpy as np
import pytest

from mfcfd_b200.batch import Batch
from mfcfd_b200.grid import batch_instances, naca_ogrid
from mfcfd_b200.solver import Solver

pytestmark = pytest.mark.gpu

BASE = dict(cfl=0.2, vl_const=5.0, power=0.0, tscheme="ssprk43")


def small_batch(inner=0, precision="fp64", tscheme="ssprk43"):
    specs = [(24, 10, 0.12, 0.6, 2.0), (40, 14, 0.10, 0.7, -1.0), (32, 12, 0.14, 0.55, 3.0),
             (64, 24, 0.12, 0.75, 0.5), (28, 10, 0.09, 0.5, 1.5)]
    grids, flows = [], []
    for k, (ni, nj, t, m, a) in enumerate(specs):
        grids.append(naca_ogrid(ni, nj, thickness=t, seed=40 + k, first_spacing=5e-3))
        flows.append(dict(BASE, mach=m, aoa=a, inner_iterations=inner, precision=precision,
                          tscheme=tscheme))
    return grids, flows


def singles(grids, flows, iters):
    out = []
    for g, f, n in zip(grids, flows, iters):
        with Solver(g, **f) as s:
            res = s.run(n)
            out.append((s.get_state(), res, s.forces()))
    return out


@pytest.mark.parametrize("inner,precision,tscheme", [(0, "fp64", "ssprk43"), (2, "fp64", "ssprk43"),
                                                     (1, "fp32_mixed", "ssprk43"),
                                                     (0, "fp64", "first")])
def test_batch_matches_single_instances(gpu, inner, precision, tscheme):
    grids, flows = small_batch(inner, precision, tscheme)
    n = 7  # odd: the graphs run iteration pairs
    ref = singles(grids, flows, [n] * len(grids))
    with Batch(grids, flows) as b:
        r = b.run(n)
        assert list(r.iters_done) == [n] * len(grids)
        assert r.state == ["max_iters"] * len(grids)
        for i, (prim, res, forces) in enumerate(ref):
            assert np.array_equal(b.get_state(i), prim), i
            assert np.array_equal(r.residue[i], res), i
            for a, c in zip(b.forces(i), forces):
                assert np.array_equal(a, c)


def test_retirement_matches_single_instances(gpu):
    grids, flows = small_batch()
    n = 40
    ref = singles(grids, flows, [n] * len(grids))
    # a tolerance the instances reach at different iterations
    tol = float(np.median([res[20] for _, res, _ in ref]))
    first = []
    for _, res, _ in ref:
        hit = np.nonzero(res <= tol)[0]
        first.append(int(hit[0]) + 1 if len(hit) else n)
    assert len(set(first)) > 1
    want = singles(grids, flows, first)
    with Batch(grids, flows) as b:
        r = b.run(n, tol=tol)
        assert list(r.iters_done) == first
        for i, (prim, res, _) in enumerate(want):
            assert r.state[i] == ("converged" if ref[i][1][first[i] - 1] <= tol else "max_iters")
            assert np.array_equal(b.get_state(i), prim), i
            assert np.array_equal(r.residue[i], res), i
        # a second call continues every instance from where it stopped
        r2 = b.run(5)
        assert list(r2.iters_done) == [5] * len(grids)
        for i, (g, f) in enumerate(zip(grids, flows)):
            with Solver(g, **f) as s:
                s.run(first[i])
                res2 = s.run(5)
                assert np.array_equal(b.get_state(i), s.get_state()), i
                assert np.array_equal(r2.residue[i], res2), i


def test_launch_shape_does_not_change_results(gpu):
    grids, flows = small_batch(inner=1)
    states = []
    for shape in [(256, 0, 0), (128, 1, 1), (128, 7, 3), (256, 100000, 100000)]:
        with Batch(grids, flows) as b:
            b.set_launch(*shape)
            r = b.run(6)
            states.append(([b.get_state(i) for i in range(len(grids))], r.residue))
    for st, res in states[1:]:
        for i in range(len(grids)):
            assert np.array_equal(st[i], states[0][0][i])
            assert np.array_equal(res[i], states[0][1][i])


def test_tuner_keeps_the_state(gpu):
    grids, flows = small_batch()
    with Batch(grids, flows) as a, Batch(grids, flows) as b:
        a.run(3)
        b.run(3)
        ms = a.tune(4)
        assert ms > 0.0
        info = a.info()
        assert info["point_block"] in (128, 256) and info["flux_grid"] >= 1
        ra, rb = a.run(4), b.run(4)
        for i in range(len(grids)):
            assert np.array_equal(a.get_state(i), b.get_state(i))
            assert np.array_equal(ra.residue[i], rb.residue[i])


def test_nonfinite_instance_retires_alone(gpu):
    grids, flows = small_batch()
    with Batch(grids, flows) as b:
        prim = b.get_state(2)
        prim[5, 0] = np.nan
        b.set_state(2, prim)
        r = b.run(6)
        assert r.status != 0
        # the residue is 0 for iterations 1 and 2, so NaN first shows at 3
        with Solver(grids[2], **flows[2]) as s:
            s.set_state(prim)
            res = s.run(6)
            assert s.halted and len(res) == 3
        assert r.state[2] == "nonfinite" and r.iters_done[2] == len(res)
        assert np.array_equal(r.residue[2], res, equal_nan=True)
        assert all(r.state[i] == "max_iters" for i in range(len(grids)) if i != 2)
        ref = singles(grids[:2], flows[:2], [6, 6])
        for i in range(2):
            assert np.array_equal(b.get_state(i), ref[i][0])


def test_set_state_round_trip(gpu):
    grids, flows = small_batch()
    rng = np.random.default_rng(0)
    with Batch(grids, flows) as b:
        for i, g in enumerate(grids):
            prim = b.get_state(i) * (1.0 + 0.01 * rng.standard_normal((g.n, 4)))
            b.set_state(i, prim)
            assert np.array_equal(b.get_state(i), prim)


def test_batched_workload_slice(gpu):
    # eight instances of the 64-instance workload (4k..60k points)
    grids, flows, _ = batch_instances(8, n_max=60000)
    ref = singles(grids, flows, [4] * len(grids))
    with Batch(grids, flows) as b:
        b.tune(2)
        r = b.run(4)
        for i, (prim, res, _) in enumerate(ref):
            assert np.array_equal(b.get_state(i), prim), i
            assert np.array_equal(r.residue[i], res), i
