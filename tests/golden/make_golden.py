"""Generates the golden fixtures under tests/golden/ from the CPU oracle.

The reference ships no golden vectors, grids or tests for this path and its
Fortran/MPI/PETSc/HDF5 toolchain is absent, so these fixtures pin the oracle
(and the CUDA path) against regression; they are not reference output.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from mfcfd_b200.grid import naca_ogrid  # noqa: E402

# name -> (grid kwargs, solver parameters, iterations)
CASES = {
    "plain": (dict(ni=40, nj=16, seed=101, first_spacing=5e-3),
              dict(cfl=0.2, vl_const=5.0, mach=0.63, aoa=2.0), 12),
    "inner3": (dict(ni=40, nj=16, seed=102, first_spacing=5e-3),
               dict(cfl=0.2, vl_const=5.0, mach=0.85, aoa=1.0, inner_iterations=3), 12),
    "first_order": (dict(ni=32, nj=14, seed=103, first_spacing=5e-3),
                    dict(cfl=0.2, vl_const=50.0, mach=0.5, aoa=-1.0, tscheme="first"), 12),
    "power_m2": (dict(ni=32, nj=14, seed=104, first_spacing=5e-3),
                 dict(cfl=0.2, vl_const=5.0, mach=0.7, aoa=3.0, power=-2.0), 12),
}


def case_grid(name):
    gk, _, _ = CASES[name]
    gk = dict(gk)
    return naca_ogrid(gk.pop("ni"), gk.pop("nj"), **gk)


def compute(name):
    gk, flow, iters = CASES[name]
    g = case_grid(name)
    o = oracle.Oracle(g, **flow)
    out = {}
    r1 = o.run(1)
    for a in ("prim", "q", "dq", "qm", "flux_res", "delta"):
        out[f"it1_{a}"] = o.get(a)
    r = o.run(iters - 1, it_first=2)
    out["residue"] = np.concatenate([r1, r])
    out["prim"] = o.prim()
    cl, cd, cm, cp = o.forces()
    out["cl"], out["cd"], out["cm"], out["cp"] = cl, cd, cm, cp
    o.close()
    return out


def main():
    for name in CASES:
        out = compute(name)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
