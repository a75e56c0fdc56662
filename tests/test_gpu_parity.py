"""Parity of the FP64 CUDA path (through the C ABI) with the CPU oracle.

Tolerances: FP64 results must agree with the oracle to 1e-10 relative in prim
after N iterations (the contract of the FP64 path), with the same residue
history (1e-9 absolute).  The remaining differences are rounding: CUDA's
exp/log/erf differ from glibc's by an ulp, and the device code contracts
a*b+c into FMA where the oracle does not.
"""
import os

import numpy as np
import pytest

import oracle
from mfcfd_b200.grid import config_flow, config_grid, naca_ogrid
from mfcfd_b200.solver import Solver
from tests.golden.make_golden import CASES, case_grid
from tests.helpers import max_rel, max_scaled

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
PRIM_RTOL = 1e-10
RES_ATOL = 1e-9


def flow_of(name):
    f = config_flow(name)
    return f


def test_stage_arrays_after_one_iteration(gpu):
    g = naca_ogrid(48, 20, seed=21, first_spacing=5e-3)
    flow = dict(cfl=0.2, vl_const=5.0, mach=0.8, aoa=1.5, inner_iterations=2)
    o = oracle.Oracle(g, **flow)
    with Solver(g, **flow) as s:
        s.keep_diagnostics(True)
        s.run(1)
        o.run(1)
        assert max_rel(s.get_array("delta"), o.get("delta")) < 1e-14
        assert max_scaled(s.get_array("q"), o.get("q")) < 1e-13
        assert max_scaled(s.get_array("dq"), o.get("dq")) < 1e-12
        assert max_scaled(s.get_array("qm"), o.get("qm")) < 1e-13
        assert max_scaled(s.get_array("flux_res"), o.get("flux_res")) < 1e-11
        assert max_rel(s.get_state(), o.prim()) < 1e-13
        assert np.allclose(s.get_array("nx"), o.get("nx"), rtol=0, atol=0)
        assert np.allclose(s.get_array("ny"), o.get("ny"), rtol=0, atol=0)


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_cases(gpu, name):
    _, flow, iters = CASES[name]
    ref = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    with Solver(case_grid(name), **flow) as s:
        s.keep_diagnostics(True)
        r1 = s.run(1)
        assert max_scaled(s.get_array("flux_res"), ref["it1_flux_res"]) < 1e-11
        assert max_scaled(s.get_array("dq"), ref["it1_dq"]) < 1e-12
        r = s.run(iters - 1)
        res = np.concatenate([r1, r])
        assert np.allclose(res, ref["residue"], rtol=0, atol=RES_ATOL)
        assert max_rel(s.get_state(), ref["prim"]) < PRIM_RTOL
        cl, cd, cm, cp = s.forces()
        assert abs(cl[0] - ref["cl"][0]) < 1e-10 and abs(cd[0] - ref["cd"][0]) < 1e-10
        assert abs(cm[0] - ref["cm"][0]) < 1e-10
        assert np.max(np.abs(cp - ref["cp"])) < 1e-10


def test_c1_full_run_matches_oracle(gpu):
    """The 16,000-point configuration for its full 1,000 iterations."""
    g = config_grid("C1")
    flow = flow_of("C1")
    o = oracle.Oracle(g, **{k: v for k, v in flow.items()})
    r_ref = o.run(1000)
    with Solver(g, **flow) as s:
        r = s.run(1000)
        prim = s.get_state()
        cl, cd, cm, _ = s.forces()
    assert len(r) == len(r_ref) == 1000
    assert np.max(np.abs(r - r_ref)) < RES_ATOL
    assert max_rel(prim, o.prim()) < PRIM_RTOL
    cl0, cd0, cm0, _ = o.forces()
    assert abs(cl[0] - cl0[0]) < 1e-10 and abs(cd[0] - cd0[0]) < 1e-10


def test_full_size_grid_two_iterations(gpu):
    """The 1,024,000-point configuration (3 inner iterations): two full
    iterations against the oracle."""
    g = config_grid("C2")
    flow = flow_of("C2")
    o = oracle.Oracle(g, **flow)
    r_ref = o.run(3)
    with Solver(g, **flow) as s:
        r = s.run(3)
        prim = s.get_state()
    assert np.max(np.abs(r - r_ref)) < RES_ATOL
    assert max_rel(prim, o.prim()) < 1e-12


def test_rcm_ordering_gives_the_same_state(gpu):
    g = naca_ogrid(64, 24, seed=31, first_spacing=5e-3)
    flow = dict(cfl=0.2, vl_const=5.0, mach=0.7, aoa=2.0, inner_iterations=1)
    with Solver(g, **flow) as a, Solver(g, ordering="rcm", **flow) as b:
        ra, rb = a.run(15), b.run(15)
        # per-point arithmetic does not depend on the numbering; only the
        # residual sum order does
        assert np.array_equal(a.get_state(), b.get_state())
        assert np.allclose(ra, rb, rtol=0, atol=1e-13)


def test_deterministic_and_chunking_invariant(gpu):
    g = naca_ogrid(64, 24, seed=32, first_spacing=5e-3)
    flow = dict(cfl=0.2, vl_const=5.0, mach=0.7, aoa=2.0, inner_iterations=3)
    with Solver(g, **flow) as a, Solver(g, **flow) as b, Solver(g, **flow) as c:
        ra = a.run(13)
        rb = np.concatenate([b.run(4), b.run(1), b.run(8)])
        rc = np.concatenate([c.run(1) for _ in range(13)])
        assert np.array_equal(ra, rb) and np.array_equal(ra, rc)
        assert np.array_equal(a.get_state(), b.get_state())
        assert np.array_equal(a.get_state(), c.get_state())


def test_nan_residue_stops_like_the_reference(gpu):
    g = naca_ogrid(32, 12, seed=5, first_spacing=5e-3)
    flow = dict(cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0)
    o = oracle.Oracle(g, **flow)
    p = o.prim()
    p[100, 3] = -1.0
    o.set_prim(p)
    r_ref = o.run(10)
    with Solver(g, **flow) as s:
        s.set_state(p)
        r = s.run(10)
        assert s.halted
        assert len(r) == len(r_ref) and np.isnan(r[-1])


def test_restart_uses_given_res_old(gpu):
    g = naca_ogrid(32, 12, seed=5, first_spacing=5e-3)
    flow = dict(cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0, restart=1, res_old=1e-3)
    o = oracle.Oracle(g, **flow)
    r_ref = o.run(3)
    with Solver(g, **flow) as s:
        r = s.run(3, it_first=1)
    assert r[0] != 0.0
    assert np.allclose(r, r_ref, rtol=0, atol=RES_ATOL)


def test_state_round_trip_and_restart_from_state(gpu):
    g = naca_ogrid(40, 16, seed=6, first_spacing=5e-3)
    flow = dict(cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0)
    with Solver(g, **flow) as a, Solver(g, **flow) as b:
        a.run(6)
        mid = a.get_state()
        b.set_state(mid)
        assert np.array_equal(b.get_state(), mid)
        a.run(4)
        b.run(4, it_first=7)
        assert np.array_equal(a.get_state(), b.get_state())


def test_mirror_symmetry_on_gpu(gpu):
    ni, nj = 48, 16
    g = naca_ogrid(ni, nj, jitter=0.0, first_spacing=5e-3)
    with Solver(g, cfl=0.2, vl_const=5.0, mach=0.6, aoa=0.0) as s:
        s.run(20)
        p = s.get_state().reshape(nj, ni, 4)
        cl = s.forces()[0]
    m = p[:, (-np.arange(ni)) % ni, :]
    assert np.max(np.abs(p[..., 0] - m[..., 0])) < 1e-12
    assert np.max(np.abs(p[..., 2] + m[..., 2])) < 1e-12
    assert abs(cl[0]) < 1e-12


def test_kernels_launched(gpu):
    g = naca_ogrid(32, 12, seed=7, first_spacing=5e-3)
    with Solver(g, cfl=0.2, vl_const=5.0, mach=0.6, aoa=1.0, inner_iterations=2) as s:
        n0 = s.launch_count()
        s.run(4)
        # per iteration: 4 stages x (grad + 2 inner + flux) + residual
        assert s.launch_count() - n0 == 4 * (4 * 4 + 1)
        t = s.profile_iteration()
        assert t["flux"] > 0 and t["iteration"] > 0
