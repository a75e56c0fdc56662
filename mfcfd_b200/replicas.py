"""Independent replicas across ranks (one process per GPU).

The pseudo-time loop shards only by domain decomposition with halo
exchanges (the reference's PETSc ghost updates), which this library leaves
out: on N GPUs it runs N independent replicas, or gives each rank every N-th
instance of a batched workload, with no exchange on the data path.  These
helpers pick a rank's share and combine per-rank results: times as the
maximum over ranks (the job ends with its slowest rank), work as the sum.
They run over whatever process group is initialised: NCCL on GPUs, gloo on
the CPU (the tests).
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> list:
    """Items of this rank: rank, rank + world, ... (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return list(range(rank, n_items, world))


def _reduce(values, op: str, dist):
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def max_over_ranks(values, dist=None) -> list:
    """Element-wise maximum over ranks (times: the slowest rank)."""
    return _reduce(values, "max", dist)


def sum_over_ranks(values, dist=None) -> list:
    """Element-wise sum over ranks (work done by the whole job)."""
    return _reduce(values, "sum", dist)
