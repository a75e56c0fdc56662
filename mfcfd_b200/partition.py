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
* ``PartitionedSolver`` runs it on the GPU (a partitioned handle iterated
  phase by phase, ghost rows refreshed between phases), and
  ``PartitionedOracle`` on the CPU oracle (test infrastructure), both
  exchanging at the reference's points.
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

def exchange_rows(rows, send: dict, recv: dict, dist, group=None):
    """Copies rows between ranks: for every peer, the rows ``send[peer]`` of
    this rank go to the peer and the rows ``recv[peer]`` are overwritten by
    what the peer sends.  Every peer pair exchanges one message each way
    (isend/irecv), so a rank never waits on a peer that waits on it.  `rows`
    is an (n, w) numpy array or torch tensor, host or device; with the gloo
    backend device rows travel through host buffers, with NCCL directly."""
    import torch
    t = torch.from_numpy(rows) if isinstance(rows, np.ndarray) else rows
    via_host = t.is_cuda and dist.get_backend(group) == "gloo"
    wire = torch.device("cpu") if via_host else t.device
    reqs, inbox, keep = [], {}, []
    for peer in sorted(set(send) | set(recv)):
        if peer in send:
            idx = torch.as_tensor(np.asarray(send[peer]), device=t.device)
            buf = t.index_select(0, idx).contiguous().to(wire)
            keep.append(buf)
            reqs.append(dist.isend(buf, peer, group=group))
        if peer in recv:
            inbox[peer] = torch.empty((len(recv[peer]),) + tuple(t.shape[1:]), dtype=t.dtype,
                                      device=wire)
            reqs.append(dist.irecv(inbox[peer], peer, group=group))
    for q in reqs:
        q.wait()
    for peer, buf in inbox.items():
        t[torch.as_tensor(np.asarray(recv[peer]), device=t.device)] = buf.to(t.device)
    return rows


def exchange(part: RankPart, rows, dist, group=None):
    """Refreshes the ghost rows of `rows` (the rank's local rows, local
    order) from their owners: VecGhostUpdate with INSERT_VALUES /
    SCATTER_FORWARD."""
    return exchange_rows(rows, part.send, part.recv, dist, group)


class _DeviceRows:
    """__cuda_array_interface__ view of rows the library owns on the device."""

    def __init__(self, ptr: int, n: int, width: int):
        self.__cuda_array_interface__ = {"shape": (n, width), "typestr": "<f8",
                                         "data": (ptr, False), "version": 3, "strides": None}


class PartitionedSolver:
    """One rank of the reference's multi-rank pseudo-time loop on the GPU: the
    rank's part as a partitioned handle (mfcfd_create_part), iterated phase
    by phase (mfcfd_part_phase) with the ghost rows refreshed between phases
    over torch.distributed (NCCL between GPUs, gloo through host buffers)
    and one all-reduce of the residual per iteration."""

    def __init__(self, part: RankPart, dist, device: int = 0, **flow):
        import ctypes as C

        import torch

        from . import _lib
        from .solver import make_params
        self.part, self.dist, self.flow = part, dist, dict(flow)
        self.torch = torch
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        self.lib = _lib.load()
        self.params = make_params(**flow)
        g = part.grid
        self._arrays = [np.ascontiguousarray(a) for a in
                        (g.x, g.y, g.nx, g.ny, g.min_dist, g.flag_1, g.flag_2, g.left, g.right,
                         g.nbhs, g.conn)]
        self._grid = _lib.Grid(g.n, *[a.ctypes.data_as(C.c_void_p) for a in self._arrays], g.n,
                               g.shapes)
        h = C.c_void_p()
        st = self.lib.mfcfd_create_part(C.byref(self._grid), C.byref(self.params), part.n_local,
                                        part.plen, C.byref(h))
        _lib.check(st, None, "mfcfd_create_part")
        self.h = h
        # one stream for the library's kernels and torch's packing: a stream
        # of its own (the default stream's handle is 0, which the library
        # reads as "keep your stream"), made torch's current stream
        self.stream = torch.cuda.Stream(self.device)
        torch.cuda.set_stream(self.stream)
        _lib.check(self.lib.mfcfd_set_stream(h, C.c_void_p(self.stream.cuda_stream)), h,
                   "mfcfd_set_stream")
        internal = np.empty(g.n, np.int32)
        _lib.check(self.lib.mfcfd_part_index(h, internal.ctypes.data_as(C.POINTER(C.c_int))), h,
                   "mfcfd_part_index")
        self.send = {k: internal[np.asarray(v)] for k, v in part.send.items()}
        self.recv = {k: internal[np.asarray(v)] for k, v in part.recv.items()}
        self.res_old = float(flow.get("res_old", 0.0))
        self.restart = int(flow.get("restart", 0))
        self._C, self._L = C, _lib

    def _phase(self, phase, rk=0, t=0):
        v = self._C.c_double(0.0)
        self._L.check(self.lib.mfcfd_part_phase(self.h, phase, rk, t, self._C.byref(v)), self.h,
                      "mfcfd_part_phase")
        return v.value

    def _refresh(self, name):
        C = self._C
        ptr, w = C.c_void_p(), C.c_int(0)
        self._L.check(self.lib.mfcfd_part_rows(self.h, name.encode(), C.byref(ptr), C.byref(w)),
                      self.h, "mfcfd_part_rows")
        rows = self.torch.as_tensor(_DeviceRows(ptr.value, self.part.grid.n, w.value),
                                    device=self.device)
        exchange_rows(rows, self.send, self.recv, self.dist)

    def run(self, n_iters: int, it_first: int = 1):
        """Runs n_iters iterations; returns the residue of each (the same on
        every rank)."""
        L = self._L
        rks = 4 if self.flow.get("tscheme", "ssprk43") == "ssprk43" else 1
        m = int(self.flow.get("inner_iterations", 0))
        out = []
        for it in range(it_first, it_first + n_iters):
            self._phase(L.PHASE_BEGIN)
            for rk in range(1, rks + 1):
                self._phase(L.PHASE_GRAD, rk)
                self._refresh("dq")
                self._refresh("qm")
                for t in range(1, m + 1):
                    self._phase(L.PHASE_INNER, rk, t)
                    self._refresh("dq")
                self._phase(L.PHASE_FLUX, rk)
                self._refresh("prim")
                self._phase(L.PHASE_GHOSTS)
            on = self.device if self.dist.get_backend() == "nccl" else "cpu"
            s = self.torch.tensor([self._phase(L.PHASE_END)], dtype=self.torch.float64,
                                  device=on)
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
        import ctypes as C
        out = np.empty((self.part.grid.n, 4))
        self._L.check(self.lib.mfcfd_get_state(self.h, out.ctypes.data_as(
            C.POINTER(C.c_double))), self.h, "mfcfd_get_state")
        return out[: self.part.n_local]

    def close(self):
        if getattr(self, "h", None):
            self.lib.mfcfd_destroy(self.h)
            self.h = None


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
