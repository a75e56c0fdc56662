"""The secondary objectives of src_mpi_primal (entropy, enstrophy,
stagnation-pressure loss) in the oracle against direct numpy restatements."""
import numpy as np

import oracle
from mfcfd_b200.grid import naca_ogrid


def test_oracle_objectives_match_the_formulas():
    g = naca_ogrid(24, 10, seed=2, first_spacing=5e-3)
    mach = 0.7
    o = oracle.Oracle(g, mach=mach, aoa=1.0, cfl=0.2, vl_const=5.0)
    o.run(6)
    rho, u1, u2, pr = o.prim().T
    gamma, pr_inf = 1.4, 1.0 / 1.4
    ent = np.abs(np.log(pr / rho ** gamma) - np.log(pr_inf)).sum()
    w = np.zeros(g.n)
    for i in range(g.n):
        k = g.conn[:g.nbhs[i], i] - 1
        dx, dy = g.x[k] - g.x[i], g.y[k] - g.y[i]
        a = np.array([[dx @ dx, dx @ dy], [dx @ dy, dy @ dy]])
        gu1 = np.linalg.solve(a, [dx @ (u1[k] - u1[i]), dy @ (u1[k] - u1[i])])
        gu2 = np.linalg.solve(a, [dx @ (u2[k] - u2[i]), dy @ (u2[k] - u2[i])])
        w[i] = gu2[0] - gu1[1]
    gp = gamma / (gamma - 1)
    p0_inf = pr_inf * (1 + 0.2 * mach * mach) ** gp
    m2 = (u1 ** 2 + u2 ** 2) / (gamma * pr / rho)
    p0 = pr * (1 + 0.2 * m2) ** gp
    stag = ((p0_inf - p0) ** 2).sum() / (p0_inf ** 2 * g.n)
    assert abs(o.objective("entropy") - ent) <= 1e-12 * ent
    assert abs(o.objective("enstrophy") - (w * w).sum()) <= 1e-9 * (w * w).sum()
    assert abs(o.objective("stagnation") - stag) <= 1e-11 * stag
    o.close()
