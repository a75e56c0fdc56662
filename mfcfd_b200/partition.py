"""Domain decomposition of a point cloud over ranks, and the ghost exchange.

The reference runs on P MPI ranks by giving each rank a group ``/<r+1>`` of
``point/point.h5``: its owned points (``local``, stencils numbered locally,
ghosts after the owned points) and its ghost points (``ghost``: PETSc global
index, x, y, min_dist; ``src_mpi_primal/point_preprocessor.F90:218,489-501``).
PETSc ghost vectors (``petsc_data_structure.F90:21-54``) number the owned
points of rank r contiguously after those of ranks < r, and
``VecGhostUpdateBegin/End(INSERT_VALUES, SCATTER_FORWARD)`` copies every
owner's rows into the ranks that hold them as ghosts -- dq and qm after the
q-derivative pass, dq after each inner iteration, prim after each stage
(``fpi_solver.F90:34-52``).

Here:

* ``partition`` splits a grid into contiguous ranges of a bandwidth-reducing
  (reverse Cuthill-McKee) order of its stencil graph, so that each rank's
  ghost layer is a thin band;
* ``RankPart`` is one rank's point set in the reference's local numbering,
  with the exchange plan (which owned rows go to which peer, which ghost rows
  come from which peer);
* ``write_partitioned_h5`` / ``read_partition_h5`` store and load the
  partition in point.h5 (one group per rank, as the reference reads it);
* ``exchange`` refreshes ghost rows over torch.distributed (gloo on the CPU,
  NCCL for device tensors): pack the send rows, isend/irecv per peer, unpack;
* ``PartitionedOracle`` runs the reference's multi-rank pseudo-time loop on
  the CPU oracle (test infrastructure), exchanging at the reference's points.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import pointh5
from .grid import INTERIOR, MAX_NBHS, Grid


@dataclasses.dataclass
class RankPart:
    rank: int
    nranks: int
    grid: Grid             # owned points then ghosts; conn/left/right in local 1-based numbers
    n_local: int           # owned points
    plen: int              # points of all ranks (the residual norm's divisor)
    offset: int            # PETSc global index (0-based) of the first owned point
    global_ids: np.ndarray  # (n,) caller-order index (0-based) of every local point
    ghost_gid: np.ndarray   # (n - n_local,) PETSc global index (0-based) of each ghost
    send: dict             # peer -> local indices (0-based) of owned rows the peer needs
    recv: dict             # peer -> local indices (0-based) of ghost rows the peer sends

    @property
    def n_ghost(self) -> int:
        return self.grid.n - self.n_local


def rcm_order(grid: Grid) -> np.ndarray:
    """Reverse Cuthill-McKee order of the symmetrised stencil graph."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    n = grid.n
    slot = np.arange(MAX_NBHS)[:, None] < grid.nbhs[None, :]
    rows = np.broadcast_to(np.arange(n)[None, :], slot.shape)[slot]
    cols = grid.conn[slot].astype(np.int64) - 1
    a = csr_matrix((np.ones(rows.size), (rows, cols)), shape=(n, n))
    return np.asarray(reverse_cuthill_mckee((a + a.T).tocsr(), symmetric_mode=True))


def _ranges(n: int, nranks: int):
    base, extra = divmod(n, nranks)
    sizes = [base + (1 if r < extra else 0) for r in range(nranks)]
    return np.concatenate(([0], np.cumsum(sizes)))


def partition(grid: Grid, nranks: int, order=None) -> list:
    """Splits `grid` over `nranks` ranks: rank r owns the r-th contiguous
    range of `order` (default: reverse Cuthill-McKee).  Ghosts are every
    stencil neighbour and ring neighbour (left/right) of an owned point that
    another rank owns, in increasing PETSc global index."""
    n = grid.n
    if nranks < 1 or nranks > max(n, 1):
        raise ValueError("nranks must be in [1, points]")
    order = rcm_order(grid) if order is None else np.asarray(order)
    bounds = _ranges(n, nranks)
    owner = np.empty(n, np.int64)
    pos = np.empty(n, np.int64)          # PETSc global index of every point
    for r in range(nranks):
        owner[order[bounds[r]:bounds[r + 1]]] = r
    pos[order] = np.arange(n)
    parts = []
    slot = np.arange(MAX_NBHS)[:, None] < grid.nbhs[None, :]
    for r in range(nranks):
        owned = order[bounds[r]:bounds[r + 1]]
        need = set(int(v) - 1 for v in grid.conn[:, owned][slot[:, owned]])
        bnd = owned[grid.flag_1[owned] != INTERIOR]
        need |= set(int(v) - 1 for v in grid.left[bnd] if v > 0)
        need |= set(int(v) - 1 for v in grid.right[bnd] if v > 0)
        ghosts = np.array(sorted((g for g in need if owner[g] != r), key=lambda g: pos[g]),
                          dtype=np.int64)
        parts.append(_rank_part(grid, r, nranks, owned, ghosts, pos[ghosts], int(bounds[r])))
    _plan_exchange(parts)
    return parts


def _rank_part(grid, r, nranks, owned, ghosts, ghost_gid, offset) -> RankPart:
    ids = np.concatenate([owned, ghosts]).astype(np.int64)
    n, nl = ids.size, owned.size
    g2l = {int(g): k for k, g in enumerate(ids)}
    conn = np.zeros((MAX_NBHS, n), np.int32)
    nb = np.zeros(n, np.int32)
    nb[:nl] = grid.nbhs[owned]
    for k, g in enumerate(owned):
        for s in range(int(grid.nbhs[g])):
            conn[s, k] = g2l[int(grid.conn[s, g]) - 1] + 1
    def ring(a):
        out = np.zeros(n, np.int32)
        for k, g in enumerate(owned):
            if a[g] > 0 and grid.flag_1[g] != INTERIOR:
                out[k] = g2l[int(a[g]) - 1] + 1
        return out
    f1 = np.full(n, INTERIOR, np.int32)
    f1[:nl] = grid.flag_1[owned]
    f2 = np.zeros(n, np.int32)
    f2[:nl] = grid.flag_2[owned]
    nx = np.zeros(n); ny = np.ones(n)
    nx[:nl], ny[:nl] = grid.nx[owned], grid.ny[owned]
    lg = Grid(x=grid.x[ids].copy(), y=grid.y[ids].copy(), nx=nx, ny=ny,
              min_dist=grid.min_dist[ids].copy(), flag_1=f1, flag_2=f2, left=ring(grid.left),
              right=ring(grid.right), nbhs=nb, conn=conn,
              original_id=grid.original_id[ids].astype(np.int32),
              qtdepth=np.zeros(n, np.int32), shapes=grid.shapes,
              name=f"{grid.name}_rank{r}of{nranks}")
    lg.validate()
    return RankPart(rank=r, nranks=nranks, grid=lg, n_local=int(nl), plen=int(grid.n),
                    offset=int(offset), global_ids=ids, ghost_gid=np.asarray(ghost_gid, np.int64),
                    send={}, recv={})


def _plan_exchange(parts):
    """Fills send/recv of every part from the ghosts' PETSc global indices:
    ghost j of rank r with global index gid is owned by rank s (offsets from
    the owned counts) at local index gid - offset_s."""
    offsets = np.array([p.offset for p in parts] + [parts[-1].offset + parts[-1].n_local])
    for p in parts:
        p.send, p.recv = {}, {}
    for p in parts:
        if p.n_ghost == 0:
            continue
        owners = np.searchsorted(offsets, p.ghost_gid, side="right") - 1
        for s in np.unique(owners):
            s = int(s)
            sel = np.nonzero(owners == s)[0]
            p.recv[s] = p.n_local + sel
            parts[s].send[p.rank] = p.ghost_gid[sel] - offsets[s]


# ---------------------------------------------------------------------------
# point.h5 with one group per rank

def write_partitioned_h5(path: str, parts) -> None:
    """Group /<r+1> per rank: owned rows with local stencil numbers (ghosts
    numbered after the owned points) and ghost rows (PETSc global index,
    1-based, x, y, min_dist)."""
    groups = []
    for p in parts:
        rows = pointh5.grid_rows(p.grid)[: p.n_local]
        g = p.grid
        ghost = np.stack([p.ghost_gid + 1.0, g.x[p.n_local:], g.y[p.n_local:],
                          g.min_dist[p.n_local:]], axis=1) if p.n_ghost else np.zeros((0, 4))
        groups.append((rows, ghost))
    pointh5.write_point_h5(path, groups)


def read_partition_h5(path: str, nranks: int, shapes: int = 1) -> list:
    """All ranks' parts of a partitioned point.h5 (x, y and min_dist of the
    ghosts from the ghost rows; the exchange plan from their global
    indices).  Each part's global_ids are PETSc global indices."""
    data = [pointh5.read_point_h5(path, r) for r in range(nranks)]
    offsets = np.concatenate(([0], np.cumsum([d["local"] for d in data])))
    plen = int(offsets[-1])
    parts = []
    for r, d in enumerate(data):
        rows, ghost = d["local_rows"], d["ghost_rows"]
        nl, ng = d["local"], d["ghost"]
        full = np.zeros((nl + ng, rows.shape[1]))
        full[:nl] = rows
        full[nl:, 0] = ghost[:, 0]
        full[nl:, 1:3] = ghost[:, 1:3]
        full[nl:, 4] = 1.0            # ny of a ghost is never read
        full[nl:, 5] = ghost[:, 3]
        full[nl:, 9] = INTERIOR
        g = pointh5.grid_from_rows(full, shapes=shapes, name=f"rank{r}")
        gid = np.concatenate([np.arange(nl) + offsets[r], ghost[:, 0].astype(np.int64) - 1])
        parts.append(RankPart(rank=r, nranks=nranks, grid=g, n_local=nl, plen=plen,
                              offset=int(offsets[r]), global_ids=gid.astype(np.int64),
                              ghost_gid=ghost[:, 0].astype(np.int64) - 1, send={}, recv={}))
    _plan_exchange(parts)
    return parts


# ---------------------------------------------------------------------------
# the exchange

def exchange(part: RankPart, rows, dist, group=None):
    """Refreshes the ghost rows of `rows` ((n, w) numpy array or torch tensor,
    the rank's local rows) from their owners: VecGhostUpdate with
    INSERT_VALUES / SCATTER_FORWARD.  Every peer pair exchanges one message
    each way (isend/irecv), so ranks never wait on a peer that waits on them."""
    import torch
    is_np = isinstance(rows, np.ndarray)
    t = torch.from_numpy(rows) if is_np else rows
    reqs, inbox = [], {}
    for peer in sorted(set(part.send) | set(part.recv)):
        if peer in part.send:
            idx = torch.as_tensor(part.send[peer], device=t.device)
            buf = t.index_select(0, idx).contiguous()
            reqs.append(dist.isend(buf, peer, group=group))
        if peer in part.recv:
            inbox[peer] = torch.empty((len(part.recv[peer]),) + tuple(t.shape[1:]),
                                      dtype=t.dtype, device=t.device)
            reqs.append(dist.irecv(inbox[peer], peer, group=group))
    for q in reqs:
        q.wait()
    for peer, buf in inbox.items():
        t[torch.as_tensor(part.recv[peer], device=t.device)] = buf
    return rows


class PartitionedOracle:
    """The reference's multi-rank pseudo-time loop (fpi_solver.F90:13-83 with
    its ghost updates) on the CPU oracle, one instance per rank.  Test
    infrastructure, as the oracle itself."""

    def __init__(self, part: RankPart, dist, **flow):
        import oracle
        self.part, self.dist = part, dist
        self.flow = flow
        self.o = oracle.Oracle(part.grid, n_local=part.n_local, plen=part.plen, **flow)
        self.res_old = float(flow.get("res_old", 0.0))
        self.restart = int(flow.get("restart", 0))

    def _refresh(self, name, width):
        a = np.ascontiguousarray(self.o.get(name).reshape(self.part.grid.n, width))
        exchange(self.part, a, self.dist)
        self.o.put(name, a)

    def run(self, n_iters: int, it_first: int = 1):
        import torch
        o = self.o
        rks = 4 if self.flow.get("tscheme", "ssprk43") == "ssprk43" else 1
        m = int(self.flow.get("inner_iterations", 0))
        self._refresh("prim", 4)
        out = []
        for it in range(it_first, it_first + n_iters):
            o.save_prim_old()
            o.func_delta()
            for rk in range(1, rks + 1):
                o.q_variables()
                o.q_derivatives()
                self._refresh("dq", 8)
                self._refresh("qm", 8)
                for _ in range(m):
                    o.q_inner_loop()
                    o.update_innerloop()
                    self._refresh("dq", 8)
                o.flux_residual()
                o.state_update(rk)
                self._refresh("prim", 4)
            s = torch.tensor([o.sum_res_sqr()], dtype=torch.float64)
            self.dist.all_reduce(s)
            res_new = float(np.sqrt(s.item())) / self.part.plen
            if it <= 2 and self.restart == 0:
                self.res_old = res_new
                residue = 0.0
            else:
                residue = float(np.log10(res_new / self.res_old))
            out.append(residue)
            if np.isnan(residue):
                break
        return np.array(out)

    def owned_prim(self):
        return self.o.prim()[: self.part.n_local]

    def close(self):
        self.o.close()
