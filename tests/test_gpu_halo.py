"""Tile halos of the D and I passes: tiles whose halo is too large to stage.

The D and I passes stage each 16-point tile's halo (the rows its points
read) in shared memory when it has at most 64 rows, and otherwise read the
tile's rows from global memory.  Grids in O-grid ring order stage every
tile; a caller whose points come in another order gives tiles with larger
halos.  These tests shuffle the caller's point order -- all of it, or a
share, so that staged and unstaged tiles meet in the same warps -- and check
the CUDA path against the oracle on the same shuffled grid (FP64: 1e-10
relative in prim, residue history 1e-9 absolute), the FP32-mixed path
against the FP64 path, and batches holding shuffled and ring-ordered
instances against single runs bit for bit; and stencils of up to 20 slots
(a point's local row bytes in three 8-byte words) against the oracle.
"""
import numpy as np
import pytest

import oracle
from mfcfd_b200.batch import Batch
from mfcfd_b200.grid import INTERIOR, OUTER, WALL, Grid, naca_ogrid
from mfcfd_b200.solver import Solver
from tests.helpers import max_rel

FLOW = dict(cfl=0.2, vl_const=5.0, mach=0.8, aoa=1.5, inner_iterations=2)
HALO_CAP, TILE = 64, 16


def permuted(g: Grid, perm: np.ndarray) -> Grid:
    """The same point cloud with point perm[j] of g as point j."""
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)

    def remap(a):  # 1-based indices, 0 = none
        a = np.asarray(a)
        return np.where(a > 0, inv[np.maximum(a, 1) - 1] + 1, 0).astype(a.dtype)

    return Grid(x=g.x[perm].copy(), y=g.y[perm].copy(), nx=g.nx[perm].copy(),
                ny=g.ny[perm].copy(), min_dist=g.min_dist[perm].copy(),
                flag_1=g.flag_1[perm].copy(), flag_2=g.flag_2[perm].copy(),
                left=remap(g.left[perm]), right=remap(g.right[perm]), nbhs=g.nbhs[perm].copy(),
                conn=np.ascontiguousarray(remap(g.conn[:, perm])),
                original_id=g.original_id[perm].copy(), qtdepth=g.qtdepth[perm].copy(),
                shapes=g.shapes, name=g.name)


def shuffled(g: Grid, frac: float, seed: int) -> Grid:
    rng = np.random.default_rng(seed)
    perm = np.arange(g.n)
    idx = np.sort(rng.choice(g.n, int(frac * g.n), replace=False))
    perm[idx] = rng.permutation(idx)
    return permuted(g, perm)


def unstaged_share(g: Grid) -> float:
    """Share of tiles whose halo exceeds the staging limit, with the library's
    renumbering (wall, outer, interior points, each in caller order)."""
    order = np.concatenate([np.where(g.flag_1 == k)[0] for k in (WALL, OUTER, INTERIOR)])
    inv = np.empty(g.n, np.int64)
    inv[order] = np.arange(g.n)
    big = 0
    ntiles = (g.n + TILE - 1) // TILE
    for t in range(ntiles):
        rows = set()
        for p in range(t * TILE, min(g.n, (t + 1) * TILE)):
            c = order[p]
            rows.add(p)
            rows.update(inv[g.conn[: g.nbhs[c], c] - 1].tolist())
        big += len(rows) > HALO_CAP
    return big / ntiles


def base_grid():
    return naca_ogrid(64, 24, seed=5, first_spacing=5e-3)


def wide_stencil_grid():
    """An O-grid whose 40 seeded interior points take their nearest other
    points up to 18-20 stencil slots: local row bytes in three words."""
    g = naca_ogrid(48, 16, seed=3, first_spacing=5e-3)
    rng = np.random.default_rng(0)
    for p in rng.choice(np.where(g.flag_1 == INTERIOR)[0], 40, replace=False):
        have = set((g.conn[: g.nbhs[p], p] - 1).tolist()) | {int(p)}
        want = 18 + int(rng.integers(0, 3))
        for k in np.argsort(np.hypot(g.x - g.x[p], g.y - g.y[p])):
            if g.nbhs[p] >= want:
                break
            if int(k) not in have:
                g.conn[g.nbhs[p], p] = k + 1
                g.nbhs[p] += 1
                have.add(int(k))
    return g


def test_ring_order_stages_every_tile():
    assert unstaged_share(base_grid()) == 0.0


def test_wide_stencils_reach_twenty_slots():
    g = wide_stencil_grid()
    assert g.nbhs.max() == 20 and int((g.nbhs >= 16).sum()) == 40


def test_shuffled_orders_give_unstaged_tiles():
    assert unstaged_share(shuffled(base_grid(), 1.0, seed=3)) > 0.9
    assert 0.1 < unstaged_share(shuffled(base_grid(), 0.05, seed=3)) < 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("frac", [1.0, 0.05])
def test_unstaged_tiles_match_the_oracle(gpu, frac):
    g = shuffled(base_grid(), frac, seed=3)
    share = unstaged_share(g)
    assert share > 0.9 if frac == 1.0 else 0.1 < share < 0.5, share
    o = oracle.Oracle(g, **FLOW)
    res_ref = o.run(6)
    with Solver(g, **FLOW) as s:
        res = s.run(6)
        assert max_rel(s.get_state(), o.prim()) < 1e-10
    o.close()
    assert np.allclose(res, res_ref, rtol=0, atol=1e-9)


@pytest.mark.gpu
def test_wide_stencils_match_the_oracle(gpu):
    g = wide_stencil_grid()
    o = oracle.Oracle(g, **FLOW)
    res_ref = o.run(6)
    with Solver(g, **FLOW) as s, Solver(g, precision="fp32_mixed", **FLOW) as s32:
        res = s.run(6)
        s32.run(6)
        assert max_rel(s.get_state(), o.prim()) < 1e-10
        assert max_rel(s32.get_state(), s.get_state()) < 1e-3
    o.close()
    assert np.allclose(res, res_ref, rtol=0, atol=1e-9)


@pytest.mark.gpu
def test_unstaged_tiles_fp32_mixed(gpu):
    g = shuffled(base_grid(), 0.05, seed=4)
    with Solver(g, **FLOW) as s64, Solver(g, precision="fp32_mixed", **FLOW) as s32:
        s64.run(20)
        s32.run(20)
        cl64, cl32 = s64.forces()[0][0], s32.forces()[0][0]
        assert abs(cl64 - cl32) < 1e-5, (cl64, cl32)
        assert max_rel(s32.get_state(), s64.get_state()) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
def test_batch_with_unstaged_tiles_matches_single_runs(gpu, precision):
    grids = [shuffled(base_grid(), 0.05, seed=6), naca_ogrid(40, 14, seed=7, first_spacing=5e-3),
             shuffled(naca_ogrid(32, 12, seed=8, first_spacing=5e-3), 1.0, seed=9)]
    flows = [dict(FLOW, precision=precision) for _ in grids]
    n = 5
    ref = []
    for g, f in zip(grids, flows):
        with Solver(g, **f) as s:
            res = s.run(n)
            ref.append((s.get_state(), res))
    with Batch(grids, flows) as b:
        r = b.run(n)
        for i, (prim, res) in enumerate(ref):
            assert np.array_equal(b.get_state(i), prim)
            assert np.array_equal(r.residue[i], res)
