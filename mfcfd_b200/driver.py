"""Host driver of a run: the reference's meshfree_solver + q_lskum sequence
(src_mpi_primal/meshfree_solver.F90:18-103, q_lskum.F90:16-79) over the C ABI.

    python -m mfcfd_b200.driver CASE_DIR

reads CASE_DIR/case.in (or input.nml), the grid CASE_DIR/point/point.h5
(group /1, the reference's reader: point_preprocessor.F90:177-546; the legacy
text CASE_DIR/point/partGrid when there is no point.h5),
optionally CASE_DIR/restart/sol.dat, runs max_iters iterations on the GPU and
writes CASE_DIR/residue, CASE_DIR/cp/cp-file, every nsave iterations
CASE_DIR/solution/sol.dat, and at the end the CUDA tree's CASE_DIR/output.dat
(with Mach number, entropy and adaptation sensor), in the reference's formats.
With ``-adjoint_mode`` in case.in it runs the reference's adjoint case instead
and writes CASE_DIR/sensitivity/sensitivity.dat.
"""
from __future__ import annotations

import os
import sys
import time

from . import io, pointh5
from .solver import Solver


def read_case_grid(case_dir: str, shapes: int = 1):
    """The case's grid: point/point.h5 as the reference reads it, else the
    legacy point/partGrid."""
    h5 = os.path.join(case_dir, "point", "point.h5")
    if os.path.exists(h5):
        return pointh5.read_grid_h5(h5, shapes=shapes)
    return io.read_partgrid(os.path.join(case_dir, "point", "partGrid"), shapes=shapes)


def run_case(case_dir: str, grid=None, quiet: bool = False, chunk: int = 100) -> dict:
    case = os.path.join(case_dir, "case.in")
    opts = io.read_case(case) if os.path.exists(case) else io.read_nml(
        os.path.join(case_dir, "input.nml"))
    params = io.solver_params(opts)
    if grid is None:
        grid = read_case_grid(case_dir, shapes=int(opts["shapes"]))
    itr, res_old = 0, 0.0
    prim0 = None
    if params["restart"]:
        itr, res_old, prim0 = io.read_restart(os.path.join(case_dir, "restart", "sol.dat"), grid.n)
        params["res_old"] = res_old
    log = (lambda *a: None) if quiet else print
    if "adjoint_mode" in opts:
        return _run_adjoint_case(case_dir, grid, params, opts, itr, res_old, prim0, log)
    t0 = time.perf_counter()
    its, res = [], []
    with Solver(grid, **params) as s:
        if prim0 is not None:
            s.set_state(prim0)
        max_iters, nsave = int(opts["max_iters"]), int(opts["nsave"])
        it = itr
        while it < itr + max_iters and not s.halted:
            # stop at each multiple of nsave to write the solution file
            n = min(chunk, itr + max_iters - it, nsave - it % nsave)
            r = s.run(n, it_first=it + 1)
            for k, v in enumerate(r):
                log(f"  iterations:{it + 1 + k:8d}       residue:{v:30.20e}")
            its.extend(range(it + 1, it + 1 + len(r)))
            res.extend(r.tolist())
            it += len(r)
            if it % nsave == 0 and not s.halted:
                io.write_solution(os.path.join(case_dir, "solution", "sol.dat"), grid,
                                  s.get_state(), it + 1, res_old)
        cl, cd, cm, cp = s.forces()
        prim = s.get_state()
        # the CUDA tree's final output (meshfree_solver.F90:100-107 of src_cuda):
        # adaptation sensor, entropy, output.dat
        mach, ent, sen, total_entropy = s.output_fields()
        io.write_output_dat(os.path.join(case_dir, "output.dat"), grid, prim, mach, ent, sen,
                            it, res_old)
    run_time = time.perf_counter() - t0
    io.write_residue(os.path.join(case_dir, "residue"), its, res)
    io.write_cp(os.path.join(case_dir, "cp", "cp-file"), grid, cp)
    log(f" Vector function is {cd[0]:.17g}")
    log(f" Run time: {run_time:.6f} seconds")
    return dict(iterations=len(res), residue=res, cl=cl, cd=cd, cm=cm, cp=cp, prim=prim,
                run_time=run_time, total_entropy=total_entropy)


def _run_adjoint_case(case_dir, grid, params, opts, itr, res_old, prim0, log) -> dict:
    """The reference's adjoint run (src_mpi_adjoint/meshfree_solver.F90:90-104):
    ``-adjoint_mode blackbox`` keeps every iteration's state, ``checkpoints``
    keeps ``-chkpts`` snapshots (q_lskum_chkpts_b.F90:65-91); dCd/dx, dCd/dy
    go to sensitivity/sensitivity.dat (post_processing.F90:41-66)."""
    max_iters = int(opts["max_iters"])
    n_rows = max_iters + 1 if opts["adjoint_mode"] == "blackbox" else int(opts.get("chkpts", 0)) + 1
    ckpt_bytes = 32 * grid.n * max(n_rows, 1)
    t0 = time.perf_counter()
    with Solver(grid, **params) as s:
        if prim0 is not None:
            s.set_state(prim0)
        J, dJdx, dJdy, n_forward = s.adjoint(max_iters, "cd", ckpt_bytes=ckpt_bytes)
        cl, cd, cm, cp = s.forces()
        prim = s.get_state()
    run_time = time.perf_counter() - t0
    it = itr + max_iters + 1
    io.write_sensitivity(os.path.join(case_dir, "sensitivity", "sensitivity.dat"), grid, dJdx,
                         dJdy, it)
    io.write_solution(os.path.join(case_dir, "solution", "sol.dat"), grid, prim, it, res_old)
    io.write_cp(os.path.join(case_dir, "cp", "cp-file"), grid, cp)
    log(f" Vector function is {J:.17g}")
    log(f" Run time: {run_time:.6f} seconds ({n_forward} forward iterations)")
    return dict(iterations=max_iters, J=J, dJdx=dJdx, dJdy=dJdy, cl=cl, cd=cd, cm=cm, cp=cp,
                prim=prim, run_time=run_time, n_forward=n_forward)


if __name__ == "__main__":
    run_case(sys.argv[1] if len(sys.argv) > 1 else ".")
