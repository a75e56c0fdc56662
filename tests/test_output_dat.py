"""The CUDA tree's output.dat (src_cuda/post_processing.F90:7-36) and its
post-processing fields, checked on the CPU: the oracle's fields against a
direct numpy restatement of the reference formulas, the file layout, and the
restart reader on it."""
import numpy as np

import oracle
from mfcfd_b200 import io
from mfcfd_b200.grid import naca_ogrid


def _fields_numpy(g, prim):
    """Straight numpy restatement of adaptation_sensors.F90:35-101,
    compute_entropy.F90:21-27 and post_processing.F90:24-27."""
    rho, u1, u2, pr = prim.T
    gamma, pr_inf = 1.4, 1.0 / 1.4
    mach = np.sqrt((u1 * u1 + u2 * u2) / np.sqrt(gamma * pr / rho))
    ent = np.abs(np.log(pr / rho ** gamma) - np.log(pr_inf))
    d2 = np.zeros(g.n)
    for i in range(g.n):
        for r in range(g.nbhs[i]):
            j = g.conn[r, i] - 1
            t1 = (rho[j] - rho[i]) * np.log((pr[i] * pr[i] * rho[j]) / (pr[j] * pr[j] * rho[i]))
            usq = (u1[j] - u1[i]) ** 2 + (u2[j] - u2[i]) ** 2
            t2 = (0.5 * rho[i] * rho[i] / pr[i]) * ((rho[j] / rho[i]) + (pr[i] * rho[j]) / (pr[j] * rho[i])) * usq
            t3 = 2 * (rho[i] * ((pr[i] * rho[j]) / (pr[j] * rho[i]) - 1)
                      + rho[j] * ((pr[j] * rho[i]) / (pr[i] * rho[j]) - 1))
            d2[i] = max(d2[i], t1 + t2 + t3)
    return mach, ent, d2 / d2.max(), ent.sum()


def test_oracle_fields_match_the_formulas():
    g = naca_ogrid(24, 10, seed=2, first_spacing=5e-3)
    o = oracle.Oracle(g, mach=0.7, aoa=1.0, cfl=0.2, vl_const=5.0)
    o.run(6)
    prim = o.prim()
    m, e, s, t = o.output_fields()
    mr, er, sr, tr = _fields_numpy(g, prim)
    np.testing.assert_allclose(m, mr, rtol=1e-13)
    np.testing.assert_allclose(e, er, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(s, sr, rtol=1e-11, atol=1e-14)
    assert abs(t - tr) <= 1e-12 * abs(tr)
    assert s.max() == 1.0 and s.min() >= 0.0


def test_output_dat_layout_and_restart(tmp_path):
    g = naca_ogrid(16, 6, seed=3, first_spacing=5e-3)
    rng = np.random.default_rng(0)
    prim = np.column_stack([1 + 0.1 * rng.random(g.n), 0.5 * rng.random(g.n),
                            0.1 * rng.random(g.n), 0.7 + 0.05 * rng.random(g.n)])
    mach, ent, sen = rng.random(g.n), rng.random(g.n), rng.random(g.n)
    path = tmp_path / "output.dat"
    io.write_output_dat(str(path), g, prim, mach, ent, sen, 250, 1.5e-3)
    lines = path.read_text().splitlines()
    assert lines[0].split()[:2] == [str(g.n), "250"]
    row = lines[1]
    assert len(row) == 2 * 30 + 2 * 4 + 7 * 30
    assert int(row[60:64]) == g.flag_1[0] and int(row[64:68]) == g.qtdepth[0]
    assert float(row[68:98]) == prim[0, 0]
    itr, res_old, back = io.read_restart(str(path), g.n)
    assert itr == 250 and res_old == 1.5e-3
    assert np.array_equal(back, prim)
