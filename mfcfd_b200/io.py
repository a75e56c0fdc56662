"""File formats of the reference around the pseudo-time loop.

* ``read_case``       PETSc options file ``case.in`` (src_mpi_primal/readcase.F90:12-125)
* ``read_nml``        CUDA-tree namelist ``input.nml`` (src_cuda/data_structure.F90:106-172)
* ``write_partgrid`` / ``read_partgrid``
                      legacy text grid ``point/partGrid`` (point_preprocessor.F90:10-150)
* ``write_residue``   ``residue`` file, one ``it residue`` line per iteration (q_lskum.F90:66)
* ``write_cp``        ``cp/cp-file``: flag_2, x, cp per shape point (compute_force_coeffs.F90:70)
* ``write_solution``  ``solution/sol.dat`` (post_processing.F90:28-34)
* ``write_sensitivity`` ``sensitivity/sensitivity.dat`` (src_mpi_adjoint/post_processing.F90:41-66)
* ``read_restart``    ``restart/sol.dat``: the primal's 9-column rows
                      (initial_conditions.F90:44-70) or the CUDA tree's 11-column
                      ``output.dat`` rows (src_mpi_adjoint/initial_conditions.F90:45-70)

Numbers are written the way gfortran's list-directed and ``e30.20`` edit
descriptors write them, so files read back with the reference's read
statements.
"""
from __future__ import annotations

import math
import os
import re

import numpy as np

from .grid import MAX_NBHS, Grid

# readcase.F90 defaults (cfl 0, max_iters 1e7, ...); Mach/aoa are the
# parameter.F90 constants of the MPI trees.
CASE_DEFAULTS = dict(cfl=0.0, mach=0.63, aoa=2.0, max_iters=10000000, tfinal=1.0e20,
                     time="steady", run_option="normal", tscheme="ssprk43", power=0.0,
                     limiter="venkat", vl_const=150.0, restart_solution="no",
                     inner_iterations=0, interior_points_normal_flag=0, shapes=1,
                     nsave=1000000, solution_accuracy="second", format_file="legacy")
_INT_KEYS = {"max_iters", "inner_iterations", "interior_points_normal_flag", "shapes", "nsave",
             "chkpts", "blockx", "blocky", "blockz"}
_REAL_KEYS = {"cfl", "mach", "aoa", "tfinal", "power", "vl_const"}


class FormatError(ValueError):
    """An input file (case.in, input.nml, partGrid, restart sol.dat) that does
    not parse: the message names the file, the line or option, and what was
    wrong.  The reference's Fortran reads stop the run on the same inputs."""


def _convert(key, value, where=""):
    try:
        if key in _INT_KEYS:
            return int(float(value.replace("d", "e").replace("D", "e")))
        if key in _REAL_KEYS:
            return float(value.replace("d", "e").replace("D", "e"))
    except ValueError:
        raise FormatError(f"{where}option -{key}: {value!r} is not a number") from None
    return value.strip().strip("'\"")


def read_case(path: str) -> dict:
    """Reads a PETSc options file: ``-key value`` pairs, '#' comments."""
    opts = dict(CASE_DEFAULTS)
    with open(path) as fh:
        text = fh.read()
    tokens = []
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if line:
            tokens.extend(line.split())
    i = 0
    while i < len(tokens):
        t = tokens[i]
        if not t.startswith("-"):
            raise FormatError(f"{path}: expected an option, got {t!r}")
        key = t.lstrip("-")
        nxt = tokens[i + 1] if i + 1 < len(tokens) else None
        if nxt is not None and (not nxt.startswith("-") or re.match(r"^-[\d.]", nxt)):
            opts[key] = _convert(key, nxt, f"{path}: ")
            i += 2
        else:
            opts[key] = True
            i += 1
    return opts


def read_nml(path: str) -> dict:
    """Reads the ``&input_parameters`` namelist of the CUDA tree."""
    opts = dict(CASE_DEFAULTS)
    opts.update(restart_solution="no", tscheme="ssprk43", format_file="legacy")
    with open(path) as fh:
        text = fh.read()
    m = re.search(r"&\s*input_parameters(.*?)/", text, re.S | re.I)
    if not m:
        raise FormatError(f"{path}: no &input_parameters group")
    for key, value in re.findall(r"(\w+)\s*=\s*('[^']*'|\"[^\"]*\"|[^,\n]+)", m.group(1)):
        opts[key.lower()] = _convert(key.lower(), value.strip().rstrip(","), f"{path}: ")
    return opts


def solver_params(opts: dict) -> dict:
    """Maps case options onto ``Solver``/``mfcfd_params`` keywords."""
    restart = str(opts.get("restart_solution", "no")) in ("same", "yes")
    return dict(cfl=float(opts["cfl"]), power=float(opts["power"]),
                vl_const=float(opts["vl_const"]), mach=float(opts["mach"]),
                aoa=float(opts["aoa"]), tscheme=str(opts["tscheme"]),
                inner_iterations=int(opts["inner_iterations"]),
                interior_points_normal_flag=int(opts["interior_points_normal_flag"]),
                format=2 if opts.get("format_file") == "quadtree" else 1,
                restart=1 if restart else 0)


# ---------------------------------------------------------------------------
# gfortran number formatting

def fortran_e(value: float, w: int = 30, d: int = 20) -> str:
    """``Ew.d`` edit descriptor: 0.ddddE+xx, right-justified in w columns."""
    v = float(value)
    if math.isnan(v):
        s = "NaN"
    elif math.isinf(v):
        s = "Infinity" if v > 0 else "-Infinity"
    elif v == 0.0:
        s = ("-" if math.copysign(1.0, v) < 0 else "") + "0." + "0" * d + "E+00"
    else:
        mant, exp = f"{abs(v):.{d - 1}e}".split("e")
        digits = mant.replace(".", "")
        e = int(exp) + 1
        sign = "-" if v < 0 else ""
        es = f"{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else f"{e:+04d}"
        s = f"{sign}0.{digits}E{es}"
    return s.rjust(w)


def fortran_list_real(v: float) -> str:
    """gfortran list-directed REAL(8): 17 significant digits, F form for
    0.1 <= |v| < 1e17, else E form, in a 25-character field plus padding."""
    v = float(v)
    if math.isnan(v):
        return "                       NaN"
    if v == 0.0 or 0.1 <= abs(v) < 1e17:
        if v == 0.0:
            body = "0.0000000000000000"
        else:
            mag = int(math.floor(math.log10(abs(v)))) + 1
            body = f"{v:.{max(17 - mag, 0)}f}"
        return body.rjust(25) + "     "
    mant, exp = f"{v:.16e}".split("e")
    e = int(exp)
    return f"{mant}E{'+' if e >= 0 else '-'}{abs(e):03d}".rjust(26)


def fortran_list_int(v: int) -> str:
    return str(int(v)).rjust(12)


# ---------------------------------------------------------------------------
# legacy partGrid text grid

def write_partgrid(grid: Grid, path: str) -> None:
    """``nproc max_points local_points ghost_points`` then one row per point:
    id x y left right flag_1 flag_2 min_dist nbhs conn(1..nbhs)."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        fh.write(f"1 {grid.n} {grid.n} 0\n")
        for k in range(grid.n):
            nb = int(grid.nbhs[k])
            conn = " ".join(str(int(c)) for c in grid.conn[:nb, k])
            fh.write(f"{int(grid.original_id[k])} {float(grid.x[k])!r} {float(grid.y[k])!r} "
                     f"{int(grid.left[k])} {int(grid.right[k])} {int(grid.flag_1[k])} "
                     f"{int(grid.flag_2[k])} {float(grid.min_dist[k])!r} {nb} {conn}\n")


def _numbers(path, lineno, tokens, kinds):
    """Converts the leading tokens of a line to the given kinds (int/float)."""
    if len(tokens) < len(kinds):
        raise FormatError(f"{path}: line {lineno}: {len(tokens)} values, expected at least "
                          f"{len(kinds)}")
    out = []
    for tok, kind in zip(tokens, kinds):
        try:
            out.append(kind(tok.replace("D", "E").replace("d", "e")) if kind is float
                       else int(tok))
        except ValueError:
            raise FormatError(f"{path}: line {lineno}: {tok!r} is not "
                              f"{'a number' if kind is float else 'an integer'}") from None
    return out


def read_partgrid(path: str, shapes: int = 1) -> Grid:
    with open(path) as fh:
        head = fh.readline().split()
        nproc, max_points, local_points, ghost_points = _numbers(path, 1, head, (int,) * 4)
        if nproc != 1:
            raise FormatError(f"{path}: check number of partitions and proc (single-rank "
                              f"reader, file has {nproc})")
        if local_points < 0 or ghost_points < 0 or max_points < local_points:
            raise FormatError(f"{path}: line 1: inconsistent point counts {head[:4]}")
        n = local_points
        x = np.zeros(n); y = np.zeros(n); md = np.zeros(n)
        left = np.zeros(n, np.int32); right = np.zeros(n, np.int32)
        f1 = np.zeros(n, np.int32); f2 = np.zeros(n, np.int32)
        nbhs = np.zeros(n, np.int32); oid = np.zeros(n, np.int32)
        conn = np.zeros((MAX_NBHS, n), np.int32)
        kinds = (int, float, float, int, int, int, int, float, int)
        for k in range(n):
            line = fh.readline()
            if not line:
                raise FormatError(f"{path}: truncated after {k} of {n} point rows")
            t = line.split()
            v = _numbers(path, k + 2, t, kinds)
            oid[k], x[k], y[k], left[k], right[k], f1[k], f2[k], md[k], nb = v
            nbhs[k] = nb
            if nb < 0 or nb > MAX_NBHS or len(t) < 9 + nb:
                raise FormatError(f"{path}: line {k + 2}: bad stencil (nbhs {nb}, "
                                  f"{len(t) - 9} indices)")
            conn[:nb, k] = _numbers(path, k + 2, t[9:9 + nb], (int,) * nb)
    g = Grid(x=x, y=y, nx=np.zeros(n), ny=np.ones(n), min_dist=md, flag_1=f1, flag_2=f2,
             left=left, right=right, nbhs=nbhs, conn=conn, original_id=oid,
             qtdepth=np.zeros(n, np.int32), shapes=shapes, name=os.path.basename(path))
    try:
        g.validate()
    except ValueError as e:
        raise FormatError(f"{path}: {e}") from None
    return g


# ---------------------------------------------------------------------------
# outputs

def write_residue(path: str, its, residues) -> None:
    with open(path, "w") as fh:
        for it, r in zip(its, residues):
            fh.write(f"{fortran_list_int(it)} {fortran_list_real(r)}\n")


def write_cp(path: str, grid: Grid, cp) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    idx = np.where(grid.flag_2 > 0)[0]
    with open(path, "w") as fh:
        for j, m in enumerate(idx):
            fh.write(f"{fortran_list_int(grid.flag_2[m])} {fortran_list_real(grid.x[m])}"
                     f"{fortran_list_real(cp[j])}\n")


def write_solution(path: str, grid: Grid, prim, it: int, res_old: float) -> None:
    """First line ``local_points, it-1, res_old`` (list-directed), then
    ``(3i8,6e30.20)`` rows: id, flag_1, flag_2, x, y, rho, u1, u2, pr."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        fh.write(f"{fortran_list_int(grid.n)}{fortran_list_int(it - 1)}{fortran_list_real(res_old)}\n")
        for i in range(grid.n):
            fh.write(f"{int(grid.original_id[i]):8d}{int(grid.flag_1[i]):8d}{int(grid.flag_2[i]):8d}"
                     + "".join(fortran_e(v) for v in (grid.x[i], grid.y[i], *prim[i])) + "\n")


def write_output_dat(path: str, grid: Grid, prim, mach, entropy, sensor, it: int,
                     res_old: float) -> None:
    """The CUDA tree's output.dat (src_cuda/post_processing.F90:7-36): first
    line ``max_points, it, res_old`` (list-directed), then
    ``(2e30.20,2i4,7e30.20)`` rows: x, y, flag_1, qtdepth, rho, u1, u2, pr,
    Mach number, entropy, sensor.  read_restart reads it back (11 columns)."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        fh.write(f"{fortran_list_int(grid.n)}{fortran_list_int(it)}{fortran_list_real(res_old)}\n")
        for i in range(grid.n):
            fh.write(fortran_e(grid.x[i]) + fortran_e(grid.y[i])
                     + f"{int(grid.flag_1[i]):4d}{int(grid.qtdepth[i]):4d}"
                     + "".join(fortran_e(v) for v in (*prim[i], mach[i], entropy[i], sensor[i]))
                     + "\n")


def write_sensitivity(path: str, grid: Grid, dJdx, dJdy, it: int) -> None:
    """``local_points, it-1`` then ``(1i8, 2e30.20)``: id, dJ/dx, dJ/dy."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        fh.write(f"{fortran_list_int(grid.n)}{fortran_list_int(it - 1)}\n")
        for i in range(grid.n):
            fh.write(f"{int(grid.original_id[i]):8d}{fortran_e(dJdx[i])}{fortran_e(dJdy[i])}\n")


def read_restart(path: str, n: int):
    """Returns (itr, res_old, prim[n,4]).  Rows of 9 values are the primal's
    sol.dat (prim in columns 6-9); rows of 11 values the CUDA tree's
    output.dat (prim in columns 5-8)."""
    with open(path) as fh:
        head = fh.readline().split()
        _, itr, res_old = _numbers(path, 1, head, (int, float, float))
        prim = np.zeros((n, 4))
        for i in range(n):
            line = fh.readline()
            if not line:
                raise FormatError(f"{path}: truncated after {i} of {n} point rows")
            t = line.split()
            if len(t) == 9:
                prim[i] = _numbers(path, i + 2, t[5:9], (float,) * 4)
            elif len(t) == 11:
                prim[i] = _numbers(path, i + 2, t[4:8], (float,) * 4)
            else:
                raise FormatError(f"{path}: line {i + 2} has {len(t)} values (want 9 or 11)")
    return int(itr), res_old, prim
