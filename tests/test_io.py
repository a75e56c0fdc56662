"""CPU tests of the reference file formats."""
import os

import numpy as np

from mfcfd_b200 import io
from mfcfd_b200.grid import naca_ogrid


def test_case_in_parsing(tmp_path):
    p = tmp_path / "case.in"
    p.write_text("-cfl 0.2\n-max_iters 2000\n-format_file legacy\n-vl_const 50\n"
                 "-inner_iterations 3\n-restart_solution no\n-power -2.0\n# comment\n")
    o = io.read_case(str(p))
    assert o["cfl"] == 0.2 and o["max_iters"] == 2000 and o["vl_const"] == 50.0
    assert o["inner_iterations"] == 3 and o["power"] == -2.0
    assert o["tscheme"] == "ssprk43" and o["mach"] == 0.63  # readcase / parameter.F90 defaults
    sp = io.solver_params(o)
    assert sp["restart"] == 0 and sp["format"] == 1


def test_nml_parsing(tmp_path):
    p = tmp_path / "input.nml"
    p.write_text("&input_parameters \n\tcfl = 0.2\n\tmax_iters = 1\n\tmach = 0.63\n"
                 "\tvl_const = 650\n\tformat_file = 'legacy'\n\ttscheme = 'ssprk43'\n"
                 "\tblockx = 32\n\tinner_iterations = 1\n\taoa = 2\n/\n")
    o = io.read_nml(str(p))
    assert o["vl_const"] == 650.0 and o["blockx"] == 32 and o["aoa"] == 2.0
    assert o["tscheme"] == "ssprk43"


def test_partgrid_round_trip(tmp_path):
    g = naca_ogrid(24, 8, seed=4)
    path = str(tmp_path / "point" / "partGrid")
    io.write_partgrid(g, path)
    h = io.read_partgrid(path)
    for name in ("x", "y", "min_dist", "flag_1", "flag_2", "left", "right", "nbhs", "conn"):
        assert np.array_equal(getattr(g, name), getattr(h, name)), name


def test_fortran_e_format():
    assert io.fortran_e(1.0) == "    0.10000000000000000000E+01"
    assert io.fortran_e(-0.125) == "   -0.12500000000000000000E+00"
    assert io.fortran_e(-0.001234) == "   -0.12340000000000000708E-02"
    assert io.fortran_e(0.0) == "    0.00000000000000000000E+00"
    assert len(io.fortran_e(3.14159)) == 30


def test_solution_and_restart_round_trip(tmp_path):
    g = naca_ogrid(24, 8, seed=4)
    rng = np.random.default_rng(0)
    prim = rng.uniform(0.5, 1.5, size=(g.n, 4))
    path = str(tmp_path / "solution" / "sol.dat")
    io.write_solution(path, g, prim, it=11, res_old=1.25e-3)
    itr, res_old, back = io.read_restart(path, g.n)
    assert itr == 10 and res_old == 1.25e-3
    assert np.max(np.abs(back - prim) / np.abs(prim)) < 1e-19 * 1e3


def test_restart_reads_cuda_output_layout(tmp_path):
    n = 3
    rows = ["3 7 1.0E-3"]
    for i in range(n):
        rows.append(f"0.1 0.2 0 0 {1 + i}.5 0.6 0.0{i} 0.7 0.5 0.0 0.0")
    p = tmp_path / "output.dat"
    p.write_text("\n".join(rows) + "\n")
    itr, res_old, prim = io.read_restart(str(p), n)
    assert itr == 7 and prim[2, 0] == 3.5 and prim[1, 2] == 0.01


def test_residue_and_cp_files(tmp_path):
    g = naca_ogrid(24, 8, seed=4)
    io.write_residue(str(tmp_path / "residue"), [1, 2, 3], [0.0, 0.0, -0.0239631])
    lines = (tmp_path / "residue").read_text().splitlines()
    assert len(lines) == 3 and lines[2].split()[0] == "3"
    assert abs(float(lines[2].split()[1]) + 0.0239631) < 1e-15
    cp = np.linspace(-1, 1, int((g.flag_2 > 0).sum()))
    io.write_cp(str(tmp_path / "cp" / "cp-file"), g, cp)
    rows = [r.split() for r in (tmp_path / "cp" / "cp-file").read_text().splitlines()]
    assert len(rows) == cp.size and int(rows[0][0]) == 1
    assert np.allclose([float(r[2]) for r in rows], cp, rtol=0, atol=1e-15)


# --- garbled and truncated inputs: each reader stops with io.FormatError ---

def test_garbled_partgrid_is_rejected(tmp_path):
    import pytest
    g = naca_ogrid(16, 6, seed=4)
    path = tmp_path / "partGrid"
    io.write_partgrid(g, str(path))
    lines = path.read_text().splitlines(keepends=True)
    cases = {
        "header_short": ["1 96 96\n"] + lines[1:],
        "header_text": ["one 96 96 0\n"] + lines[1:],
        "two_ranks": ["2 96 96 0\n"] + lines[1:],
        "counts": ["1 10 96 0\n"] + lines[1:],
        "truncated": lines[:40],
        "row_text": lines[:5] + [lines[5].replace(lines[5].split()[1], "x.y", 1)] + lines[6:],
        "row_short": lines[:7] + ["7 0.1 0.2 0 0\n"] + lines[8:],
        "stencil": lines[:9] + [" ".join(lines[9].split()[:8] + ["25"]) + "\n"] + lines[10:],
        "conn_range": lines[:3] + [" ".join(lines[3].split()[:9] + ["999"] * int(lines[3].split()[8]))
                                   + "\n"] + lines[4:],
    }
    for name, text in cases.items():
        p = tmp_path / f"pg_{name}"
        p.write_text("".join(text))
        with pytest.raises(io.FormatError, match=str(p)):
            io.read_partgrid(str(p))


def test_garbled_restart_is_rejected(tmp_path):
    import pytest
    g = naca_ogrid(16, 6, seed=4)
    prim = np.tile([1.0, 0.5, 0.0, 1 / 1.4], (g.n, 1))
    path = tmp_path / "sol.dat"
    io.write_solution(str(path), g, prim, 11, 1e-3)
    it, res_old, back = io.read_restart(str(path), g.n)
    assert it == 10 and res_old == 1e-3 and np.array_equal(back, prim)
    lines = path.read_text().splitlines(keepends=True)
    cases = {
        "header_text": ["96 ten 1e-3\n"] + lines[1:],
        "truncated": lines[:50],
        "row_width": lines[:4] + [" ".join(lines[4].split()[:7]) + "\n"] + lines[5:],
        "row_text": lines[:4] + [lines[4].replace(lines[4].split()[6], "nanx", 1)] + lines[5:],
    }
    for name, text in cases.items():
        p = tmp_path / f"sol_{name}.dat"
        p.write_text("".join(text))
        with pytest.raises(io.FormatError, match=str(p)):
            io.read_restart(str(p), g.n)


def test_garbled_case_files_are_rejected(tmp_path):
    import pytest
    bad = {
        "value": "-cfl fast\n-max_iters 10\n",
        "int": "-inner_iterations three\n",
        "token": "cfl 0.2\n",
    }
    for name, text in bad.items():
        p = tmp_path / f"case_{name}.in"
        p.write_text(text)
        with pytest.raises(io.FormatError, match=str(p)):
            io.read_case(str(p))
    p = tmp_path / "input.nml"
    p.write_text("&other_group\n cfl = 0.2\n/\n")
    with pytest.raises(io.FormatError, match="no &input_parameters"):
        io.read_nml(str(p))
    p.write_text("&input_parameters\n cfl = abc\n/\n")
    with pytest.raises(io.FormatError, match="-cfl"):
        io.read_nml(str(p))
