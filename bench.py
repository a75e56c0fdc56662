#!/usr/bin/env python3
"""Throughput benchmark of the LSKUM pseudo-time loop on B200.

One step is one pseudo-time iteration (fpi_solver: local time step, four
SSPRK stages with 3 inner least-squares iterations each, residual) over the
1280 x 800 = 1,024,000-point NACA 0012 O-grid at M = 0.85, aoa = 1 deg in
FP64 -- the workload the headline metric is quoted on.  Grids are synthetic
(seeded), since the reference ships none.

  value     device-timed throughput, state resident in HBM (CUDA events on the
            stream the library launches on)
  e2e       the same through the C ABI with host buffers: set_state from host,
            one mfcfd_run call per step (its residue copied back each step),
            get_state + forces at the end -- all inside the timed region
  roofline  the flux kernel (the dominant one): algorithmic bytes per launch
            over its CUDA-event duration, against the measured HBM copy peak
  cpu_baseline  the oracle (C restatement of src_mpi_primal) on the host's
            cores, on a bounded sample of the same workload
  fp32_mixed, adjoint, batch  the FP32-mixed loop on the same workload, the
            reverse-mode cost against the primal, and the 64-instance batched
            workload against one handle at a time
  adjoint_batch  the adjoint of Cd over 16 instances of 16k-1M points in one
            mfcfd_adjoint_many call against one mfcfd_adjoint at a time

``--impl reference`` times that CPU restatement alone (the reference itself
is Fortran + MPI + PETSc + HDF5 and cannot be built on these machines).
Under torchrun each rank runs an independent replica (the loop is
single-GPU); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mfcfd_b200.replicas import max_over_ranks, shard, sum_over_ranks  # noqa: E402

METRIC = "Mpoint-iters/s @1M pts FP32-mix vs FP64 at |ΔCl|≤1e-5; adjoint/primal cost"
UNIT = "Mpoint-iters/s"
FALLBACK_HBM_GBS = 6650.0


def workload_config(name: str, grid, flow: dict) -> dict:
    from mfcfd_b200.grid import CONFIGS
    c = CONFIGS[name]
    return {
        "workload": (f"{name}: NACA 0012 O-grid {c['ni']}x{c['nj']} = {grid.n:,} points, "
                     f"M={flow['mach']}, aoa={flow['aoa']} deg, {flow['inner_iterations']} inner "
                     f"LSQ iterations, SSPRK(4,3), CFL {flow['cfl']}, Venkat K={flow['vl_const']}, FP64"),
        "points": grid.n,
        "mean_stencil": round(grid.mean_nbhs(), 4),
        "inner_iterations": flow["inner_iterations"],
        "l2": "no flush: the per-iteration working set (~0.45 GB at 1M points) exceeds the 126 MB L2",
    }


def algorithmic_bytes(kbar: float, m: int, rks: int = 4) -> dict:
    """Minimal dataflow bytes per point: each pass reads and writes every
    array it touches once (split lists derive from conn).  The I pass in its
    rearranged form reads the D pass's dq0 (64 B) in place of q (32 B)."""
    t = 92 + 4 * kbar
    d = 180 + 4 * kbar
    i = 212 + 4 * kbar
    f = 280 + 4 * kbar
    return {"flux_pass": f, "grad_pass": d, "inner_pass": i, "step_pass": t,
            "iteration": t + rks * (d + m * i + f)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh)
    return {}


def _profile_value(key: str):
    """A figure of the committed ncu summary of kb_flux (``key: value`` line)."""
    p = os.path.join(ROOT, "profiles", "kb_flux_fp64_c2.md")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        for line in fh:
            m = re.match(r"\s*" + key + r":\s*([0-9.eE+]+)", line)
            if m:
                return float(m.group(1))
    return None


def profiled_traffic(workload: str):
    """dram bytes per launch of kb_flux from the committed ncu summary."""
    return _profile_value("dram_bytes_per_launch_full_size")


def fp64_peak_tflops():
    """FP64 FMA throughput of the current device (library kernel), TFLOP/s."""
    import ctypes
    from mfcfd_b200 import _lib
    v = ctypes.c_double(0.0)
    if _lib.load().mfcfd_measure_fp64_peak(ctypes.byref(v)) != _lib.MFCFD_OK:
        return None
    return v.value


class ClockSampler:
    """nvidia-smi clocks during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return None
        self.file.flush()
        with open(self.file.name) as fh:
            rows = [r.split(",") for r in fh.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(grid, flow: dict, budget_s: float, rank0: bool = True) -> dict:
    """Times the oracle on the host cores: iterations of the full grid until
    about ``budget_s`` seconds of CPU work."""
    import oracle
    f = dict(flow)
    f.pop("tscheme", None)
    o = oracle.Oracle(grid, **f)
    threads = oracle.num_threads()
    t0 = time.perf_counter()
    o.run(1, it_first=1)
    first = time.perf_counter() - t0
    n_more = max(1, min(200, int(budget_s / max(first, 1e-3)) - 1))
    t0 = time.perf_counter()
    o.run(n_more, it_first=2)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": grid.n * n_more / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"{n_more} pseudo-time iterations of the full {grid.n:,}-point grid "
                       f"(after 1 warm-up iteration), oracle C restatement of src_mpi_primal, "
                       f"OpenMP over points, {threads} threads, {dt:.1f} s")}


def run_reference(args, grid, flow, cfg):
    """--impl reference: the CPU restatement timed step by step."""
    import oracle
    f = dict(flow)
    f.pop("tscheme", None)
    o = oracle.Oracle(grid, **f)
    threads = oracle.num_threads()
    it = 1
    for _ in range(args.warmup):
        o.run(1, it_first=it)
        it += 1
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.run(1, it_first=it)
        it += 1
    dt = time.perf_counter() - t0
    value = grid.n * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": (f"each step one pseudo-time iteration of the full {grid.n:,}-point "
                                    f"grid; oracle C restatement of src_mpi_primal (the Fortran/MPI/"
                                    f"PETSc/HDF5 reference cannot be built here), {threads} threads")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def adjoint_cost(args, stream, world, dist):
    """Adjoint/primal cost on the adjoint configuration (640 x 400 = 256,000
    points, M 0.63, aoa 2 deg): a state developed for --adjoint-develop
    iterations is held fixed; the primal run of n iterations from it and the
    reverse-mode gradient over the same n iterations are device-timed on the
    same stream, for J = Cd and J = Cl with binomial checkpoints of prim
    within the configured 2 GB (--adjoint-ckpt-bytes), and for J = Cd once
    more with a snapshot of every iteration (32 B a point per iteration, 16.4
    GB here: each iteration then runs forward once and once more taped).
    Each handle allocates its tape and snapshot pool on its first call,
    inside that call's time (one allocation each)."""
    import torch
    from mfcfd_b200.grid import config_flow, config_grid
    from mfcfd_b200.solver import Solver
    grid = config_grid(args.adjoint_config)
    flow = config_flow(args.adjoint_config)
    n = args.adjoint_iters
    budget = args.adjoint_ckpt_bytes
    budget_all = (n + 1) * 32 * grid.n
    # untimed warm-up: the first call of a kernel in a process loads its module
    from mfcfd_b200.grid import naca_ogrid
    with Solver(naca_ogrid(32, 12, seed=1, first_spacing=5e-3), **flow) as w:
        w.set_stream(stream.cuda_stream)
        w.adjoint(2, "cd")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Solver(grid, **flow) as s:
        s.set_stream(stream.cuda_stream)
        s.run(args.adjoint_develop)
        start = s.get_state()
        torch.cuda.synchronize()
        e0.record(stream)
        s.run(n)
        e1.record(stream)
        torch.cuda.synchronize()
        primal_ms = e0.elapsed_time(e1)
        out = {}
        for key, obj, b in (("cd", "cd", budget), ("cl", "cl", budget),
                            ("cd_all", "cd", budget_all)):
            s.set_state(start)
            torch.cuda.synchronize()
            e0.record(stream)
            J, dx, dy, nf = s.adjoint(n, obj, ckpt_bytes=b)
            e1.record(stream)
            torch.cuda.synchronize()
            out[key] = (e0.elapsed_time(e1), J, nf,
                        float(max(np.abs(dx).max(), np.abs(dy).max())))
    primal_ms, cd_ms, cl_ms, all_ms = max_over_ranks(
        [primal_ms, out["cd"][0], out["cl"][0], out["cd_all"][0]], dist)
    return {"config": (f"{args.adjoint_config}: {grid.n:,} points, M {flow['mach']}, aoa "
                       f"{flow['aoa']} deg, {n} iterations reversed from a state developed for "
                       f"{args.adjoint_develop}, prim snapshots within "
                       f"{budget / 2**30:.1f} GiB"),
            "primal_ms": primal_ms,
            "adjoint_ms": {"cd": cd_ms, "cl": cl_ms},
            "cost_ratio": cd_ms / primal_ms, "cost_ratio_cl": cl_ms / primal_ms,
            "forward_iterations": out["cd"][2], "checkpoint_budget_bytes": budget,
            "all_snapshots": {"checkpoint_budget_bytes": budget_all, "adjoint_ms_cd": all_ms,
                              "cost_ratio": all_ms / primal_ms,
                              "forward_iterations": out["cd_all"][2]},
            "J": {"cd": out["cd"][1], "cl": out["cl"][1]},
            "grad_max": {"cd": out["cd"][3], "cl": out["cl"][3]}}


def fp32_accuracy(grid, flow: dict, n_iters: int, stream, label: str) -> dict:
    """The FP32-mixed loop against the FP64 loop after n_iters iterations from
    freestream on the same grid: Cl, Cd and prim (RMS and max of the
    difference relative to max(|prim|, 1e-3 max|prim| of the component))."""
    from mfcfd_b200.solver import Solver
    with Solver(grid, **flow) as a, Solver(grid, precision="fp32_mixed", **flow) as b:
        a.set_stream(stream.cuda_stream)
        b.set_stream(stream.cuda_stream)
        ra, rb = a.run(n_iters), b.run(n_iters)
        if len(ra) != n_iters or len(rb) != n_iters:
            return {"config": label, "iterations": n_iters, "nonfinite": True,
                    "iterations_done": [len(ra), len(rb)]}
        pa, pb = a.get_state(), b.get_state()
        cla, cda, _, _ = a.forces()
        clb, cdb, _, _ = b.forces()
    scale = np.maximum(np.abs(pa), 1e-3 * np.max(np.abs(pa), axis=0))
    err = np.abs(pb - pa) / scale
    return {"config": label, "iterations": n_iters,
            "dCl": abs(float(clb[0] - cla[0])), "dCd": abs(float(cdb[0] - cda[0])),
            "Cl_fp64": float(cla[0]), "Cd_fp64": float(cda[0]),
            "prim_rms_rel": float(np.sqrt(np.mean(err ** 2))), "prim_max_rel": float(err.max()),
            "residue_fp64": float(ra[-1]), "residue_fp32": float(rb[-1])}


def adjoint_batch_leg(args, world, rank, dist):
    """The batched adjoint: 16 seeded instances of 16k-1M points (thickness,
    M and aoa drawn per instance as for the batched primal), sharded across
    ranks, each developed for the warm-up iterations and then reversed over
    n iterations for J = Cd (2 GB of snapshots each).  Timed twice from the
    same states, after an untimed call that allocates every buffer: one
    mfcfd_adjoint per instance in turn, and one mfcfd_adjoint_many call
    (instances under 65,536 points overlap the others on their own streams
    and host threads).  Both calls are
    synchronous, so each is timed on the host around the call (gradients to
    host included); max over ranks."""
    import torch
    from mfcfd_b200.grid import batch_instances, naca_ogrid
    from mfcfd_b200.solver import Solver, adjoint_many
    grids, flows, _ = batch_instances(args.adjoint_batch_instances, config=5, n_min=16000,
                                      n_max=1_000_000)
    mine = shard(len(grids), rank, world)
    grids, flows = [grids[i] for i in mine], [flows[i] for i in mine]
    n = args.adjoint_batch_iters
    budget = 2 << 30
    with Solver(naca_ogrid(32, 12, seed=1, first_spacing=5e-3), **flows[0]) as w:
        w.adjoint(2, "cd")  # untimed: module loading
    solvers = [Solver(g, **f) for g, f in zip(grids, flows)]
    try:
        for s in solvers:
            s.run(args.warmup)
        start = [s.get_state() for s in solvers]
        # untimed: allocates every handle's tape and snapshot pool, so that
        # neither timed pass pays for allocation
        adjoint_many(solvers, n, "cd", ckpt_bytes=budget)
        for s, p in zip(solvers, start):
            s.set_state(p)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        single = [s.adjoint(n, "cd", ckpt_bytes=budget) for s in solvers]
        seq_s = time.perf_counter() - t0
        for s, p in zip(solvers, start):
            s.set_state(p)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        many = adjoint_many(solvers, n, "cd", ckpt_bytes=budget)
        many_s = time.perf_counter() - t0
        same = all(np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and a[0] == b[0]
                   for a, b in zip(single, many))
    finally:
        for s in solvers:
            s.close()
    seq_s, many_s = max_over_ranks([seq_s, many_s], dist)
    points = sum_over_ranks([sum(g.n for g in grids)], dist)[0]
    return {"config": (f"{args.adjoint_batch_instances} NACA 00tt O-grids, N log-uniform in "
                       f"[16k, 1M] (seeded draws), M in [0.5, 0.8], aoa in [-2, 4] deg, t in "
                       f"[0.08, 0.16], FP64, J = Cd, {n} iterations reversed each"),
            "instances_per_rank": len(grids), "points": int(points),
            "one_call_s": many_s, "one_handle_at_a_time_s": seq_s,
            "speedup_vs_one_at_a_time": seq_s / many_s,
            "value": points * n / many_s / 1e6, "unit": "Mpoint-iters reversed/s",
            "bitwise_equal_to_single": bool(same)}


def batch_leg(args, stream, world, rank, dist):
    """The batched workload: 64 seeded instances (4k-256k points, M, aoa and
    thickness drawn per instance; FP32-mixed unless --batch-precision says
    otherwise), sharded across ranks with no exchange,
    advanced together by one Batch for a bounded number of iterations (tol
    -8 retires an instance early), device-timed on the stream; beside it the
    same instances run one Solver at a time for the same iterations."""
    import torch
    from mfcfd_b200.batch import Batch
    from mfcfd_b200.grid import batch_instances
    from mfcfd_b200.solver import Solver
    grids, flows, specs = batch_instances(args.batch_instances)
    mine = shard(len(grids), rank, world)
    grids = [grids[i] for i in mine]
    flows = [dict(flows[i], precision=args.batch_precision) for i in mine]
    n = args.batch_iters
    with Batch(grids, flows) as b:
        b.set_stream(stream.cuda_stream)
        tuned_ms = b.tune(4)
        b.run(args.warmup)
        torch.cuda.synchronize()
        l0 = b.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = b.run(n, tol=-8.0)
        e1.record(stream)
        torch.cuda.synchronize()
        batch_ms = e0.elapsed_time(e1)
        launches = b.launch_count() - l0
        info = b.info()
    work = sum(g.n * int(d) for g, d in zip(grids, r.iters_done))
    seq_ms = 0.0
    for g, f, d in zip(grids, flows, r.iters_done):
        with Solver(g, **f) as s:
            s.set_stream(stream.cuda_stream)
            s.run(args.warmup)
            torch.cuda.synchronize()
            e0.record(stream)
            s.run(int(d))
            e1.record(stream)
            torch.cuda.synchronize()
            seq_ms += e0.elapsed_time(e1)
    batch_ms, seq_ms = max_over_ranks([batch_ms, seq_ms], dist)
    work = sum_over_ranks([work], dist)[0]
    states = {k: r.state.count(k) for k in sorted(set(r.state))}
    return {"config": (f"{args.batch_instances} NACA 00tt O-grids, N log-uniform in [4k, 256k] "
                       f"(seeded draws), M in [0.5, 0.8], aoa in [-2, 4] deg, t in [0.08, 0.16], "
                       f"{args.batch_precision}, retire at residue <= -8 or {n} iterations"),
            "instances_per_rank": len(grids), "points_per_rank": int(sum(g.n for g in grids)),
            "iterations": n, "value": work / (batch_ms / 1e3) / 1e6, "unit": UNIT,
            "ms": batch_ms, "one_handle_at_a_time_ms": seq_ms,
            "speedup_vs_one_at_a_time": seq_ms / batch_ms, "states_rank0": states,
            "gpu_launches": launches, "launch_shape": info, "tuner_ms_per_iter": tuned_ms}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("mfcfd", "reference"), default="mfcfd")
    ap.add_argument("--config", default="C2")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--fp32-check-iters", type=int, default=300,
                    help="iterations from freestream after which the FP32-mixed loop is "
                         "compared with the FP64 loop on the bench grid (0 = skip)")
    ap.add_argument("--adjoint-iters", type=int, default=2000,
                    help="iterations reversed by the adjoint-cost leg (0 = skip)")
    ap.add_argument("--adjoint-develop", type=int, default=1000,
                    help="iterations that develop the adjoint leg's starting state")
    ap.add_argument("--adjoint-config", default="C3")
    ap.add_argument("--adjoint-ckpt-bytes", type=int, default=2 << 30,
                    help="snapshot budget of the adjoint leg (the configuration's 2 GB)")
    ap.add_argument("--batch-iters", type=int, default=100,
                    help="iterations of the batched-workload leg (0 = skip)")
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--batch-precision", choices=("fp32_mixed", "fp64"), default="fp32_mixed",
                    help="precision of the batched leg (the batched workload is FP32-mixed)")
    ap.add_argument("--adjoint-batch-iters", type=int, default=20,
                    help="iterations reversed by the batched-adjoint leg (0 = skip)")
    ap.add_argument("--adjoint-batch-instances", type=int, default=16)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "mfcfd":
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    from mfcfd_b200.grid import config_flow, config_grid
    if args.impl == "reference":
        if rank != 0:
            return
        grid = config_grid(args.config)
        flow = config_flow(args.config)
        run_reference(args, grid, flow, workload_config(args.config, grid, flow))
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from mfcfd_b200.solver import Solver
    grid = config_grid(args.config)
    flow = config_flow(args.config)
    cfg = workload_config(args.config, grid, flow)
    parallelism = f"replicas x{world}" if world > 1 else "single GPU"
    f = dict(flow)
    solver = Solver(grid, **f)
    stream = torch.cuda.Stream()
    solver.set_stream(stream.cuda_stream)

    solver.run(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = solver.launch_count()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        t_start.record(stream)
        res = solver.run(args.steps)
        t_end.record(stream)
        torch.cuda.synchronize()
    launches = solver.launch_count() - launches0
    if solver.halted or len(res) != args.steps:
        raise RuntimeError(f"FP64 run stopped on a non-finite residue after {len(res)} of "
                           f"{args.steps} timed iterations: no throughput to report")
    ms = t_start.elapsed_time(t_end)
    ms = max_over_ranks([ms], dist)[0]
    if dist:
        dist.barrier()
    clocks = clk.summary()
    value = world * grid.n * args.steps / (ms / 1e3) / 1e6
    cl64, cd64, _, _ = solver.forces()
    it64 = solver.it

    # FP32-mixed: same grid, same number of iterations, device-timed the same way
    fp32 = None
    if not args.no_fp32:
        s32 = Solver(grid, precision="fp32_mixed", **f)
        s32.set_stream(stream.cuda_stream)
        s32.run(args.warmup)
        torch.cuda.synchronize()
        f_start = torch.cuda.Event(enable_timing=True)
        f_end = torch.cuda.Event(enable_timing=True)
        f_start.record(stream)
        res32 = s32.run(args.steps)
        f_end.record(stream)
        torch.cuda.synchronize()
        ms32 = f_start.elapsed_time(f_end)
        ms32 = max_over_ranks([ms32], dist)[0]
        halted32 = bool(s32.halted) or len(res32) != args.steps
        cl32, cd32, _, _ = s32.forces()
        kt32 = {} if halted32 else s32.profile_iteration()
        s32.close()
        v32 = world * grid.n * args.steps / (ms32 / 1e3) / 1e6
        # the FP32-mixed flux pass against HBM: the FP64 pass table with the
        # five FP32-stored state arrays (prim, prim_old, q, dq, qm) at 4
        # bytes (280 - 112 = 168) plus the 8-byte slot offsets it stores
        f32_bytes_pt = 168 + 12 * grid.mean_nbhs()
        f32_roof = None
        if kt32.get("flux"):
            ach32 = f32_bytes_pt * grid.n / (kt32["flux"] / 1e3) / 1e9
            peak32 = measured_peaks().get("hbm_gbs", FALLBACK_HBM_GBS)
            f32_roof = {"kernel": "kb_flux32", "bound": "hbm", "algorithmic_bytes_per_point":
                        f32_bytes_pt, "achieved": ach32, "peak": peak32, "unit": "GB/s",
                        "frac": ach32 / peak32}
        fp32 = {"value": v32, "unit": UNIT, "ms_per_step": ms32 / args.steps,
                "speedup_vs_fp64": v32 / value, "iterations": it64, "roofline": f32_roof,
                "dCl": abs(float(cl32[0] - cl64[0])), "dCd": abs(float(cd32[0] - cd64[0])),
                "Cl_fp64": float(cl64[0]), "Cd_fp64": float(cd64[0]),
                "kernel_ms": {k: float(v) for k, v in kt32.items()},
                "note": "FP32 state, fluxes and Kahan sums; the state update's arithmetic, "
                        "the geometry (LSQ inverses, formed once), the residual and the "
                        "forces in FP64; dCl/dCd against the FP64 run after the same "
                        "iterations, 'accuracy' after --fp32-check-iters from freestream"}
        if args.fp32_check_iters > 0 and not halted32:
            fp32["accuracy"] = fp32_accuracy(grid, f, args.fp32_check_iters, stream,
                                             cfg["workload"].split(":")[0])
        if halted32:
            fp32.update(value=None, speedup_vs_fp64=None, ms_per_step=None,
                        nonfinite=True, iterations_done=len(res32),
                        note="FP32-mixed run stopped on a non-finite residue")

    # per-kernel CUDA-event durations on the same stream (extra iterations)
    prof = [solver.profile_iteration() for _ in range(3)]
    kt = {k: float(np.mean([p[k] for p in prof])) for k in prof[0]}
    ab = algorithmic_bytes(grid.mean_nbhs(), flow["inner_iterations"])
    peaks = measured_peaks()
    peak = peaks.get("hbm_gbs", FALLBACK_HBM_GBS)
    flux_bytes = ab["flux_pass"] * grid.n
    achieved = flux_bytes / (kt["flux"] / 1e3) / 1e9
    traffic = profiled_traffic(args.config)
    hbm_roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "algorithmic_bytes_per_launch": flux_bytes,
                "peak_source": ("MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks
                                else "fallback 6.65 TB/s")}
    # The binding roof of the flux pass is FP64 issue: its FP64 work per
    # point (flop-equivalents, FMA = 2, from the executed DFMA/DMUL/DADD
    # counts of the committed ncu capture) over the kernel's CUDA-event time,
    # against the FP64 FMA peak measured on this device by the library.
    fp64_peak = fp64_peak_tflops()
    flops_pt = _profile_value("fp64_flops_per_point")
    roofline = dict(hbm_roof)
    if fp64_peak and flops_pt:
        fp64_achieved = flops_pt * grid.n / (kt["flux"] / 1e3) / 1e12
        roofline = {"bound": "fp64", "achieved": fp64_achieved, "peak": fp64_peak,
                    "unit": "TFLOP/s", "frac": fp64_achieved / fp64_peak, "traffic": traffic,
                    "fp64_flops_per_point": flops_pt,
                    "peak_source": "mfcfd_measure_fp64_peak (FMA chains, this device)",
                    "hbm": hbm_roof}
    roofline.update({
        "kernel": "kb_flux (flux residual + state update, one SSPRK stage)",
        "fp64_pipe_active_frac": _profile_value("fp64_pipe_active_frac"),
        "note": ("kb_flux is bound by FP64 latency (exp/erf/div chains), not by HBM: "
                 "achieved/peak is its FP64 work rate against the measured FMA peak; "
                 "the hbm object gives its algorithmic bytes against the copy peak")})
    iter_bytes = ab["iteration"] * grid.n
    iteration_roof = {"algorithmic_bytes_per_iteration": iter_bytes,
                      "achieved_gbs": iter_bytes / (ms / args.steps / 1e3) / 1e9,
                      "hbm_roof_mpt_it_s": peak * 1e9 / ab["iteration"] / 1e6}

    e2e = None
    if not args.no_e2e:
        host_prim = np.ascontiguousarray(solver.get_state())
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        e_start = torch.cuda.Event(enable_timing=True)
        e_end = torch.cuda.Event(enable_timing=True)
        e_start.record(stream)
        solver.set_state(host_prim)
        for _ in range(args.steps):
            solver.run(1)
        out_prim = solver.get_state()
        cl, cd, cm, cp = solver.forces()
        e_end.record(stream)
        torch.cuda.synchronize()
        e_ms = e_start.elapsed_time(e_end)
        wall_ms = (time.perf_counter() - t0) * 1e3
        e_ms = max(e_ms, wall_ms)
        e_ms = max_over_ranks([e_ms], dist)[0]
        state_bytes = 32 * grid.n
        e2e = {"value": world * grid.n * args.steps / (e_ms / 1e3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": 8 + (state_bytes + 8 * (3 + cp.size)) / args.steps,
               "timed": ("set_state from host, one mfcfd_run per step (residue to host each "
                         "step), get_state + forces at the end")}

    adjoint = None
    if args.adjoint_iters > 0:
        adjoint = adjoint_cost(args, stream, world, dist)

    batch = None
    if args.batch_iters > 0:
        batch = batch_leg(args, stream, world, rank, dist)

    adjoint_batch = None
    if args.adjoint_batch_iters > 0:
        adjoint_batch = adjoint_batch_leg(args, world, rank, dist)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(grid, flow, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg, "parallelism": parallelism,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks,
            "kernel_ms": kt, "iteration_roofline": iteration_roof,
            "final_residue": float(res[-1]) if len(res) else None,
            "fp32_mixed": fp32,
            "adjoint": adjoint,
            "batch": batch,
            "adjoint_batch": adjoint_batch,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
