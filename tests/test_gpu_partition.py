"""The partitioned GPU loop (mfcfd_create_part + mfcfd_part_phase, ghost rows
refreshed between phases over torch.distributed) against the single-grid
loop.  Ranks run as spawned processes on the one visible GPU and exchange
through gloo host buffers, so no kernel waits on another process.  Each
owned point's arithmetic is the single-grid kernels' on identical inputs:
the state is bit for bit the same; only the residual's sum order differs."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from mfcfd_b200 import partition as PT
from mfcfd_b200.grid import naca_ogrid

pytestmark = pytest.mark.gpu
FLOW = dict(cfl=0.2, vl_const=5.0, mach=0.7, aoa=1.5, inner_iterations=2)
N_ITERS = 7


def _grid():
    return naca_ogrid(64, 24, seed=31, first_spacing=5e-3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = PT.partition(_grid(), world)
        ps = PT.PartitionedSolver(parts[rank], dist, **FLOW)
        res = ps.run(N_ITERS)
        out[rank] = dict(res=res, ids=parts[rank].global_ids[: parts[rank].n_local],
                         prim=ps.owned_prim(), nghost=parts[rank].n_ghost)
        ps.close()
    finally:
        dist.destroy_process_group()


def _run_ranks(world):
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        return [dict(out[k]) for k in range(world)]


@pytest.mark.parametrize("world", [1, 2])
def test_partitioned_gpu_loop_matches_the_single_grid_loop(gpu, world):
    from mfcfd_b200.solver import Solver
    r = _run_ranks(world)
    g = _grid()
    with Solver(g, **FLOW) as s:
        res = s.run(N_ITERS)
        prim = s.get_state()
    merged = np.full_like(prim, np.nan)
    for x in r:
        merged[x["ids"]] = x["prim"]
        assert np.array_equal(x["res"], r[0]["res"])
    if world > 1:
        assert all(x["nghost"] > 0 for x in r)
    assert np.array_equal(merged, prim)
    assert np.allclose(r[0]["res"], res, rtol=0, atol=1e-13)
