"""The multi-rank path on the CPU: two gloo ranks shard the batched workload
and combine their times and work the way bench.py does on N GPUs (no GPU
needed: the per-rank work is the oracle on a small grid)."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from mfcfd_b200.grid import batch_instances
from mfcfd_b200.replicas import max_over_ranks, shard, sum_over_ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _, _, specs = batch_instances(64, build=False)
        mine = shard(len(specs), rank, world)
        points = sum(specs[i]["ni"] * specs[i]["nj"] for i in mine)
        everyone = [None] * world
        dist.all_gather_object(everyone, mine)
        # a replica's work: a few oracle iterations on a small grid
        import oracle
        from mfcfd_b200.grid import naca_ogrid
        o = oracle.Oracle(naca_ogrid(24, 10, seed=rank + 1, first_spacing=5e-3), mach=0.6)
        res = o.run(3)
        o.close()
        t_max = max_over_ranks([1.0 + rank, 10.0 * (world - rank)], dist)
        work = sum_over_ranks([points, len(res)], dist)
        out[rank] = dict(everyone=everyone, t_max=t_max, work=work, points=points,
                         total=sum(s["ni"] * s["nj"] for s in specs))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    # spawn, not fork: the test process may already hold CUDA or other threads
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        r0, r1 = dict(out[0]), dict(out[1])
    shards = r0["everyone"]
    assert shards == r1["everyone"]
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(64))                        # every instance once
    assert not set(shards[0]) & set(shards[1])
    assert r0["t_max"] == r1["t_max"] == [2.0, 20.0]      # the slowest rank
    assert r0["work"][0] == r0["total"]                   # all points counted once
    assert r0["work"][1] == 6                             # 3 iterations per rank


def test_single_process_helpers():
    assert shard(5, 0, 1) == [0, 1, 2, 3, 4]
    assert shard(5, 1, 2) == [1, 3]
    assert max_over_ranks([1.5, 2.0]) == [1.5, 2.0]
    assert np.allclose(sum_over_ranks([3, 4]), [3.0, 4.0])
