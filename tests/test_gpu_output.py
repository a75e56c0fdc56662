"""mfcfd_output_fields (the CUDA tree's Mach / entropy / D2-sensor columns of
output.dat) against the oracle on the same state."""
import numpy as np
import pytest

import oracle
from mfcfd_b200.grid import naca_ogrid
from mfcfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
def test_output_fields_match_the_oracle(gpu, precision):
    g = naca_ogrid(48, 16, seed=4, first_spacing=5e-3)
    flow = dict(cfl=0.2, vl_const=5.0, mach=0.7, aoa=1.5, precision=precision)
    with Solver(g, **flow) as s:
        s.run(8)
        prim = s.get_state()
        m, e, sen, tot = s.output_fields()
    flow.pop("precision")
    o = oracle.Oracle(g, **flow)
    o.set_prim(prim)
    mr, er, sr, tr = o.output_fields()
    o.close()
    np.testing.assert_allclose(m, mr, rtol=1e-13)
    np.testing.assert_allclose(e, er, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(sen, sr, rtol=1e-11, atol=1e-14)
    assert abs(tot - tr) <= 1e-12 * abs(tr)


def test_driver_runs_a_case_directory(gpu, tmp_path):
    # meshfree_solver's sequence over the C ABI: case.in + point/partGrid in,
    # residue, cp/cp-file, solution/sol.dat (every nsave) and output.dat out
    from mfcfd_b200 import io
    from mfcfd_b200.driver import run_case
    g = naca_ogrid(32, 12, seed=9, first_spacing=5e-3)
    (tmp_path / "point").mkdir()
    io.write_partgrid(g, str(tmp_path / "point" / "partGrid"))
    (tmp_path / "case.in").write_text("-cfl 0.2\n-max_iters 12\n-vl_const 5\n-nsave 5\n"
                                      "-mach 0.63\n-aoa 2.0\n")
    out = run_case(str(tmp_path), quiet=True, chunk=4)
    assert out["iterations"] == 12
    with Solver(io.read_partgrid(str(tmp_path / "point" / "partGrid")), cfl=0.2, vl_const=5.0,
                mach=0.63, aoa=2.0) as s:
        res = s.run(12)
        assert np.array_equal(out["prim"], s.get_state())
    r = np.loadtxt(tmp_path / "residue")
    assert r.shape == (12, 2) and np.allclose(r[:, 1], res, rtol=1e-14, atol=1e-300)
    itr, _, prim10 = io.read_restart(str(tmp_path / "solution" / "sol.dat"), g.n)
    assert itr == 10
    itr, _, prim12 = io.read_restart(str(tmp_path / "output.dat"), g.n)
    assert itr == 12 and np.array_equal(prim12, out["prim"])
    assert (tmp_path / "cp" / "cp-file").exists()


@pytest.mark.parametrize("mode", ["blackbox", "checkpoints"])
def test_driver_runs_an_adjoint_case(gpu, tmp_path, mode):
    # src_mpi_adjoint's run: -adjoint_mode, -chkpts; sensitivity/sensitivity.dat out
    from mfcfd_b200 import io
    from mfcfd_b200.driver import run_case
    g = naca_ogrid(24, 10, seed=10, first_spacing=5e-3)
    (tmp_path / "point").mkdir()
    io.write_partgrid(g, str(tmp_path / "point" / "partGrid"))
    (tmp_path / "case.in").write_text(f"-cfl 0.2\n-max_iters 6\n-vl_const 5\n-adjoint_mode {mode}\n"
                                      "-chkpts 2\n")
    out = run_case(str(tmp_path), quiet=True)
    gg = io.read_partgrid(str(tmp_path / "point" / "partGrid"))
    with Solver(gg, cfl=0.2, vl_const=5.0) as s:
        J, dx, dy, nf = s.adjoint(6, "cd")
    assert out["J"] == J
    rows = np.loadtxt(tmp_path / "sensitivity" / "sensitivity.dat", skiprows=1)
    assert np.array_equal(rows[:, 0].astype(int), np.arange(1, g.n + 1))
    np.testing.assert_allclose(rows[:, 1], dx, rtol=1e-15, atol=0)
    np.testing.assert_allclose(rows[:, 2], dy, rtol=1e-15, atol=0)
    assert (out["n_forward"] > nf) == (mode == "checkpoints")
