"""Point-cloud grids in the reference's point layout.

The reference reads a point cloud per rank from ``point/point.h5`` (group
``/1``, dataset ``local`` with one row per point: id, x, y, nx, ny, min_dist,
left, right, qtdepth, flag_1, flag_2, nbhs, conn...;
``src_mpi_primal/point_preprocessor.F90:353-371``) or from the legacy text file
``point/partGrid`` (``point_preprocessor.F90:56-60``).  It ships no grid, so
this module also generates the synthetic NACA 00tt O-grids the benchmarks run
on.

Arrays use the reference's conventions: point numbers are 1-based, ``conn`` is
the Fortran ``conn(N,20)`` array stored column-major (``conn[r-1, i-1]`` in the
``(20, N)`` numpy array is slot r of point i), 0 marks an unused slot.
flag_1: 0 wall, 1 interior, 2 outer.  flag_2: shape number (0 = not on a shape).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

MAX_NBHS = 20
WALL, INTERIOR, OUTER = 0, 1, 2


@dataclasses.dataclass
class Grid:
    x: np.ndarray          # (N,) f64
    y: np.ndarray          # (N,) f64
    nx: np.ndarray         # (N,) f64  (file normals; legacy format overrides them)
    ny: np.ndarray         # (N,) f64
    min_dist: np.ndarray   # (N,) f64
    flag_1: np.ndarray     # (N,) i32
    flag_2: np.ndarray     # (N,) i32
    left: np.ndarray       # (N,) i32, 1-based, 0 for interior points
    right: np.ndarray      # (N,) i32
    nbhs: np.ndarray       # (N,) i32
    conn: np.ndarray       # (20, N) i32, 1-based; memory order == Fortran conn(N,20)
    original_id: np.ndarray  # (N,) i32
    qtdepth: np.ndarray      # (N,) i32
    shapes: int = 1
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def mean_nbhs(self) -> float:
        return float(self.nbhs.mean()) if self.n else 0.0

    def validate(self) -> None:
        """Structural checks the reader performs (shapes, index ranges)."""
        n = self.n
        for name in ("x", "y", "nx", "ny", "min_dist"):
            a = getattr(self, name)
            if a.shape != (n,) or a.dtype != np.float64:
                raise ValueError(f"grid.{name}: expected ({n},) float64")
        for name in ("flag_1", "flag_2", "left", "right", "nbhs", "original_id", "qtdepth"):
            a = getattr(self, name)
            if a.shape != (n,) or a.dtype != np.int32:
                raise ValueError(f"grid.{name}: expected ({n},) int32")
        if self.conn.shape != (MAX_NBHS, n) or self.conn.dtype != np.int32:
            raise ValueError(f"grid.conn: expected ({MAX_NBHS}, {n}) int32")
        if n == 0:
            return
        if self.nbhs.min() < 0 or self.nbhs.max() > MAX_NBHS:
            raise ValueError("nbhs out of range [0, 20]")
        slot = np.arange(MAX_NBHS)[:, None] < self.nbhs[None, :]
        used = self.conn[slot]
        if used.size and (used.min() < 1 or used.max() > n):
            raise ValueError("conn index out of range")
        if np.any(~np.isin(self.flag_1, (WALL, INTERIOR, OUTER))):
            raise ValueError("flag_1 must be 0, 1 or 2")
        if self.flag_2.max(initial=0) > self.shapes:
            raise ValueError("shapes value wrong, check again")
        bnd = self.flag_1 != INTERIOR
        for name in ("left", "right"):
            a = getattr(self, name)[bnd]
            if a.size and (a.min() < 1 or a.max() > n):
                raise ValueError(f"{name} index out of range on a boundary point")


def naca_thickness(x: np.ndarray, t: float) -> np.ndarray:
    """NACA 4-digit half thickness with the closed-trailing-edge coefficient."""
    x = np.clip(x, 0.0, 1.0)
    return 5.0 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x**2
                      + 0.2843 * x**3 - 0.1036 * x**4)


def _stretch_ratio(length: np.ndarray, d1, nseg: int) -> np.ndarray:
    """Solve d1 * (r**nseg - 1)/(r - 1) = length for r > 1, per ray (bisection)."""
    lo = np.full_like(length, 1.0 + 1e-12)
    hi = np.full_like(length, 2.0)
    def f(r):
        with np.errstate(over="ignore"):
            return d1 * np.expm1(nseg * np.log(r)) / (r - 1.0) - length
    while np.any(f(hi) < 0):
        hi = np.where(f(hi) < 0, hi * 2.0, hi)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        neg = f(mid) < 0
        lo = np.where(neg, mid, lo)
        hi = np.where(neg, hi, mid)
    return 0.5 * (lo + hi)


def reference_normals(g: "Grid", interior_points_normal_flag: int = 0):
    """Normals as the reference sets them (point_normals.F90:8-105, legacy format)."""
    nx = np.zeros(g.n)
    ny = np.ones(g.n)
    if interior_points_normal_flag == 1:
        nx[:], ny[:] = 1.0, 0.0
    b = np.where(g.flag_1 != INTERIOR)[0]
    l, r = g.left[b] - 1, g.right[b] - 1
    ax = 0.5 * ((g.y[b] - g.y[l]) + (g.y[r] - g.y[b]))
    ay = 0.5 * ((g.x[b] - g.x[l]) + (g.x[r] - g.x[b]))
    det = np.sqrt(ax * ax + ay * ay)
    nx[b], ny[b] = -ax / det, ay / det
    return nx, ny


def _split_membership(kind, ds, dn):
    """Membership of neighbours in xpos, xneg, ypos, yneg
    (generate_connectivity.F90:39-256); kind 0 wall, 1 interior, 2 outer."""
    ones = np.ones_like(ds, dtype=bool)
    none = np.zeros_like(ds, dtype=bool)
    ypos = np.where(kind == INTERIOR, dn <= 0, np.where(kind == OUTER, ones, none))
    yneg = np.where(kind == INTERIOR, dn >= 0, np.where(kind == WALL, ones, none))
    return [ds <= 0, ds >= 0, ypos, yneg]


def split_conditioning(g: "Grid", chunk: int = 1 << 20):
    """Relative determinant det/(sum dels^2 + sum deln^2)^2 of each point's
    four split-list LSQ matrices (inf for lists the point type does not use)
    and the list sizes.  A value near 0 means a singular flux derivative."""
    nx, ny = reference_normals(g)
    kmax = int(g.nbhs.max(initial=0))
    rel = np.full((g.n, 4), np.inf)
    cnt = np.zeros((g.n, 4), dtype=np.int32)
    for a in range(0, g.n, chunk):
        b = min(g.n, a + chunk)
        pts = np.arange(a, b)
        slot = np.arange(kmax)[:, None] < g.nbhs[None, a:b]
        idx = np.where(slot, g.conn[:kmax, a:b] - 1, 0)
        dx, dy = g.x[idx] - g.x[pts], g.y[idx] - g.y[pts]
        tx, ty = ny[a:b], -nx[a:b]
        ds, dn = dx * tx + dy * ty, dx * nx[a:b] + dy * ny[a:b]
        kind = g.flag_1[None, a:b]
        for d, m in enumerate(_split_membership(kind, ds, dn)):
            m = m & slot
            sa = np.where(m, ds * ds, 0).sum(0)
            sb = np.where(m, dn * dn, 0).sum(0)
            sab = np.where(m, ds * dn, 0).sum(0)
            sc = (sa + sb) ** 2
            used = np.where(g.flag_1[a:b] == WALL, d != 2,
                            np.where(g.flag_1[a:b] == OUTER, d != 3, True))
            val = np.where(sc > 0, (sa * sb - sab * sab) / np.where(sc > 0, sc, 1.0), 0.0)
            rel[a:b, d] = np.where(used, val, np.inf)
            cnt[a:b, d] = m.sum(0)
    return rel, cnt


def _list_rel_det(g, p, d, tx, ty, nx, ny, extra=None):
    """Relative determinant of list d of point p, with point ``extra``
    (0-based) appended to the stencil when given."""
    nb = g.conn[:g.nbhs[p], p] - 1
    if extra is not None:
        nb = np.append(nb, extra)
    dx, dy = g.x[nb] - g.x[p], g.y[nb] - g.y[p]
    ds, dn = dx * tx + dy * ty, dx * nx + dy * ny
    m = _split_membership(np.full(nb.shape, g.flag_1[p]), ds, dn)[d]
    sa, sb, sab = (ds[m] ** 2).sum(), (dn[m] ** 2).sum(), (ds[m] * dn[m]).sum()
    sc = (sa + sb) ** 2
    return (sa * sb - sab * sab) / sc if sc > 0 else 0.0


def _augment_stencils(g: "Grid", ni: int, nj: int, min_rel: float) -> int:
    """Adds neighbours to points whose split lists are singular.

    For each list whose relative determinant is below ``min_rel`` the nearest
    points of the (i+-w, j+-2) block (w = 3, then 8, then 16) that fall into
    that list under the reference's split rule are appended one at a time
    until the list is well-posed.  Returns the number of points changed."""
    rel, _ = split_conditioning(g)
    bad = np.where((rel < min_rel).any(1))[0]
    if bad.size == 0:
        return 0
    nx, ny = reference_normals(g)
    for p in bad:
        p = int(p)
        j, i = divmod(p, ni)
        tx, ty = ny[p], -nx[p]
        for d in range(4):
            if (g.flag_1[p] == WALL and d == 2) or (g.flag_1[p] == OUTER and d == 3):
                continue
            for w in (3, 8, 16):
                if _list_rel_det(g, p, d, tx, ty, nx[p], ny[p]) >= min_rel:
                    break
                cand = {jj * ni + (i + di) % ni for jj in range(max(0, j - 2), min(nj, j + 3))
                        for di in range(-w, w + 1)}
                cand = np.array(sorted(cand - {p}), dtype=np.int64)
                cdx, cdy = g.x[cand] - g.x[p], g.y[cand] - g.y[p]
                cds, cdn = cdx * tx + cdy * ty, cdx * nx[p] + cdy * ny[p]
                inlist = _split_membership(np.full(cand.shape, g.flag_1[p]), cds, cdn)[d]
                order = [c for c in np.argsort(np.hypot(cdx, cdy), kind="stable") if inlist[c]]
                for c in order:
                    if _list_rel_det(g, p, d, tx, ty, nx[p], ny[p]) >= min_rel:
                        break
                    if g.nbhs[p] >= MAX_NBHS:
                        break
                    if (g.conn[:g.nbhs[p], p] == cand[c] + 1).any():
                        continue
                    g.conn[g.nbhs[p], p] = cand[c] + 1
                    g.nbhs[p] += 1
    return int(bad.size)


def _repair_stencils(g: "Grid", ni: int, nj: int, min_rel: float) -> int:
    """Rebuilds the stencils that _augment_stencils left singular.

    Nearest-first filling fails where every close candidate of a list lies on
    one line through the point: at the wall points next to a sharp trailing
    edge, whose (i, j>=1) neighbours all sit behind them along straight rays,
    so that one list holds only (collinear) wall points while the others use
    up the MAX_NBHS slots.  Such a point restarts from its base stencil (8
    interior, 5 ring) and, while a used list is below ``min_rel``, gives the
    worst list one point of the (i+-w, j+-3) block (w = 3, 8, 16, 32, 48):
    the nearest candidate that makes the list well-posed, else the one that
    raises its relative determinant most (at least tenfold).  Points whose
    lists were all well-posed after the first pass are left untouched.
    Returns the number of points rebuilt."""
    rel, _ = split_conditioning(g)
    bad = np.where((rel < min_rel).any(1))[0]
    if bad.size == 0:
        return 0
    nx, ny = reference_normals(g)
    for p in bad:
        p = int(p)
        j, i = divmod(p, ni)
        tx, ty = ny[p], -nx[p]
        base = 8 if g.flag_1[p] == INTERIOR else 5
        g.conn[base:, p] = 0
        g.nbhs[p] = base
        lists = [d for d in range(4)
                 if not ((g.flag_1[p] == WALL and d == 2) or (g.flag_1[p] == OUTER and d == 3))]
        given_up = set()
        while g.nbhs[p] < MAX_NBHS:
            cur = {d: _list_rel_det(g, p, d, tx, ty, nx[p], ny[p])
                   for d in lists if d not in given_up}
            low = [d for d in cur if cur[d] < min_rel]
            if not low:
                break
            d = min(low, key=lambda e: cur[e])
            present = set((g.conn[:g.nbhs[p], p] - 1).tolist())
            pick = None
            for w in (3, 8, 16, 32, 48):
                cand = {jj * ni + (i + di) % ni for jj in range(max(0, j - 3), min(nj, j + 4))
                        for di in range(-w, w + 1)}
                cand = np.array(sorted(cand - {p} - present), dtype=np.int64)
                cdx, cdy = g.x[cand] - g.x[p], g.y[cand] - g.y[p]
                cds, cdn = cdx * tx + cdy * ty, cdx * nx[p] + cdy * ny[p]
                inlist = _split_membership(np.full(cand.shape, g.flag_1[p]), cds, cdn)[d]
                order = [c for c in np.argsort(np.hypot(cdx, cdy), kind="stable") if inlist[c]]
                if not order:
                    continue
                after = [_list_rel_det(g, p, d, tx, ty, nx[p], ny[p], cand[c]) for c in order]
                good = [k for k, a in enumerate(after) if a >= min_rel]
                if good:
                    pick = cand[order[good[0]]]
                    break
                best = int(np.argmax(after))
                if after[best] > 10.0 * max(cur[d], 0.0) and after[best] > 1e-8:
                    pick = cand[order[best]]
                    break
            if pick is None:
                given_up.add(d)
                continue
            g.conn[g.nbhs[p], p] = pick + 1
            g.nbhs[p] += 1
    return int(bad.size)


def naca_ogrid(ni: int, nj: int, thickness: float = 0.12, radius: float = 20.0,
               first_spacing: float = 1e-3, jitter: float = 0.1, seed: int = 0,
               name: str = "", spacing: str = "cosine", rays: str = "straight",
               augment: bool = True, min_rel_det: float = 1e-4) -> Grid:
    """NACA 00tt O-grid point cloud of ni (around) x nj (radial) points.

    Ring j=0 is the airfoil (flag_1=0, flag_2=1) with ``spacing`` "cosine"
    (clustered at both ends), "halfcos" (clustered at the leading edge) or
    "arc" (uniform in arc length on each surface);
    ring j=nj-1 a circle of ``radius`` chords about (0.5, 0) (flag_1=2).
    Points on both rings run clockwise in i (i=0 is the trailing edge), so
    ``right`` is the next point clockwise and the reference's normal formula
    points out of the body and out of the domain.  Radial spacing grows
    geometrically from ``first_spacing`` (ratio solved per ray); "match"
    makes it, per ray, the wall spacing at the ray's foot, so that the cells
    next to the wall are near-square.  ``rays``
    "straight" joins wall point i to outer point i; "blend" leaves the wall
    along the wall normal on the rounded front and turns to the straight line
    towards the trailing edge and the outer circle.  Interior points are
    jittered uniformly by +-``jitter`` of the local min(radial,
    circumferential) spacing, drawn from numpy's PCG64 with ``seed``.
    Stencils: interior 8 (i+-1, j+-1 and diagonals, periodic in i);
    wall/outer 5 (ring neighbours + 3 on the adjacent ring).  With
    ``augment`` a point whose split list (under the reference's split rule)
    is singular -- relative determinant below ``min_rel_det`` -- gets the
    nearest extra points of its (i+-3, j+-2) block appended until the list is
    well-posed; near the sharp trailing edge this is unavoidable with a fixed
    8/5 stencil.  A point still singular after that is rebuilt by
    _repair_stencils (worst list first, from a wider block).  Point ids run
    1..N in (j, i) order.
    """
    if ni < 4 or nj < 3:
        raise ValueError("naca_ogrid needs ni >= 4 and nj >= 3")
    phi = 2.0 * math.pi * np.arange(ni) / ni
    if spacing == "cosine":
        xw = 0.5 * (1.0 + np.cos(phi))
    elif spacing == "halfcos":
        xw = 1.0 - np.cos(0.5 * math.pi * np.abs(1.0 - phi / math.pi))
    elif spacing == "arc":
        if ni % 2:
            raise ValueError("spacing 'arc' needs an even ni")
        h = ni // 2
        xs = 0.5 * (1.0 + np.cos(np.linspace(0.0, math.pi, 20001)))  # TE -> LE
        cum = np.concatenate(([0.0], np.cumsum(np.hypot(np.diff(xs),
                                                       np.diff(naca_thickness(xs, thickness))))))
        xh = np.interp(np.linspace(0.0, cum[-1], h + 1), cum, xs)
        xw = np.empty(ni)
        xw[:h + 1] = xh
        xw[h + 1:] = xh[1:h][::-1]
    else:
        raise ValueError(f"unknown spacing {spacing!r}")
    yt = naca_thickness(xw, thickness)
    yw = np.where(phi < math.pi, -yt, yt)
    yw[0] = 0.0
    xo = 0.5 + radius * np.cos(phi)
    yo = -radius * np.sin(phi)
    # the trailing- and leading-edge rays lie exactly on y = 0 (sin(pi) is
    # not 0 in floating point; a 1e-15 tilt would put their on-ray neighbours
    # in one y split list instead of both)
    on_axis = (np.arange(ni) == 0) | (2 * np.arange(ni) == ni)
    yo[on_axis] = 0.0
    yw[on_axis] = 0.0
    dxr, dyr = xo - xw, yo - yw
    length = np.hypot(dxr, dyr)
    if isinstance(first_spacing, str):
        if first_spacing != "match":
            raise ValueError(f"unknown first_spacing {first_spacing!r}")
        # per ray: the mean of the two wall segments at the ray's foot
        seg = np.hypot(np.roll(xw, -1) - xw, np.roll(yw, -1) - yw)
        d1 = 0.5 * (seg + np.roll(seg, 1))
    else:
        d1 = np.full(ni, float(first_spacing))
    r = _stretch_ratio(length, d1, nj - 1)
    j = np.arange(nj)[:, None]
    s = d1[None, :] * np.expm1(j * np.log(r)[None, :]) / (r[None, :] - 1.0)
    s[-1, :] = length
    frac = s / length[None, :]
    ex, ey = dxr / length, dyr / length
    if rays == "straight":
        X = xw[None, :] + s * ex[None, :]
        Y = yw[None, :] + s * ey[None, :]
    elif rays == "smooth":
        # Ray direction b: the outward wall normal averaged over a window of
        # ni/32 rays each side, so the rays fan out gradually around the
        # sharp trailing edge instead of leaving it almost tangent to the
        # surface; the ray bends from b to the straight line as in "blend".
        tdx, tdy = np.roll(xw, -1) - np.roll(xw, 1), np.roll(yw, -1) - np.roll(yw, 1)
        tn = np.hypot(tdx, tdy)
        nwx, nwy = -tdy / tn, tdx / tn
        wdw = max(2, ni // 32)
        bx = sum(np.roll(nwx, m) for m in range(-wdw, wdw + 1))
        by = sum(np.roll(nwy, m) for m in range(-wdw, wdw + 1))
        bn = np.hypot(bx, by)
        bx, by = bx / bn, by / bn
        lam = 0.5
        off = lam * (-np.expm1(-s / lam)) * (1.0 - frac)
        X = xw[None, :] + s * ex[None, :] + off * (bx - ex)[None, :]
        Y = yw[None, :] + s * ey[None, :] + off * (by - ey)[None, :]
    elif rays == "blend":
        # Ray direction b: the wall normal over the rounded front, turning to
        # the straight line towards the sharp trailing edge.  Along a ray the
        # point is W + s e + (b - e) lam (1 - exp(-s/lam)) (1 - s/L): it
        # leaves the wall along b, ends on the outer circle, and stays within
        # lam |b - e| of the straight ray.
        wdx, wdy = np.roll(xw, -1) - np.roll(xw, 1), np.roll(yw, -1) - np.roll(yw, 1)
        wn = np.hypot(wdx, wdy)
        w = np.clip((1.0 - xw) / 0.4, 0.0, 1.0) ** 2
        bx, by = w * (-wdy / wn) + (1.0 - w) * ex, w * (wdx / wn) + (1.0 - w) * ey
        bn = np.hypot(bx, by)
        bx, by = bx / bn, by / bn
        lam = 0.5
        off = lam * (-np.expm1(-s / lam)) * (1.0 - frac)
        X = xw[None, :] + s * ex[None, :] + off * (bx - ex)[None, :]
        Y = yw[None, :] + s * ey[None, :] + off * (by - ey)[None, :]
    else:
        raise ValueError(f"unknown rays {rays!r}")
    X[-1, :], Y[-1, :] = xo, yo
    if ni % 2 == 0:
        # exact mirror symmetry about y = 0 before jitter: points that are
        # aligned in exact arithmetic stay aligned (their dels/deln tie at 0
        # and they enter both split lists on both sides)
        h = ni // 2
        X[:, h + 1:] = X[:, 1:h][:, ::-1]
        Y[:, h + 1:] = -Y[:, 1:h][:, ::-1]
        Y[:, 0] = 0.0
        Y[:, h] = 0.0

    if jitter > 0 and nj > 2:
        def dist(ax, ay, bx, by):
            return np.hypot(ax - bx, ay - by)
        jj = slice(1, nj - 1)
        rad = np.minimum(dist(X[2:], Y[2:], X[jj], Y[jj]), dist(X[jj], Y[jj], X[:-2], Y[:-2]))
        circ = np.minimum(dist(np.roll(X[jj], -1, 1), np.roll(Y[jj], -1, 1), X[jj], Y[jj]),
                          dist(np.roll(X[jj], 1, 1), np.roll(Y[jj], 1, 1), X[jj], Y[jj]))
        h = np.minimum(rad, circ)
        rng = np.random.Generator(np.random.PCG64(seed))
        u = rng.uniform(-1.0, 1.0, size=(nj - 2, ni, 2))
        X[jj] = X[jj] + jitter * h * u[..., 0]
        Y[jj] = Y[jj] + jitter * h * u[..., 1]

    n = ni * nj
    pid = (np.arange(nj)[:, None] * ni + np.arange(ni)[None, :])  # 0-based (j,i)
    ip = lambda a: np.roll(a, -1, axis=1)   # i+1
    im = lambda a: np.roll(a, 1, axis=1)    # i-1
    conn = np.zeros((MAX_NBHS, nj, ni), dtype=np.int64)
    nbhs = np.zeros((nj, ni), dtype=np.int32)
    # interior rows
    inner = slice(1, nj - 1)
    lower, upper = pid[0:nj - 2], pid[2:nj]
    mid = pid[inner]
    for slot, arr in enumerate((im(lower), lower, ip(lower), im(mid), ip(mid),
                                im(upper), upper, ip(upper))):
        conn[slot, inner] = arr + 1
    nbhs[inner] = 8
    # wall ring (j = 0) and outer ring (j = nj-1)
    for jr, jadj in ((0, 1), (nj - 1, nj - 2)):
        ring, adj = pid[jr], pid[jadj]
        for slot, arr in enumerate((np.roll(ring, 1), np.roll(ring, -1),
                                    np.roll(adj, 1), adj, np.roll(adj, -1))):
            conn[slot, jr] = arr + 1
        nbhs[jr] = 5

    flat_conn = conn.reshape(MAX_NBHS, n).astype(np.int32)
    flag_1 = np.full((nj, ni), INTERIOR, dtype=np.int32)
    flag_1[0], flag_1[-1] = WALL, OUTER
    flag_2 = np.zeros((nj, ni), dtype=np.int32)
    flag_2[0] = 1
    left = np.zeros((nj, ni), dtype=np.int32)
    right = np.zeros((nj, ni), dtype=np.int32)
    for jr in (0, nj - 1):
        left[jr] = np.roll(pid[jr], 1) + 1
        right[jr] = np.roll(pid[jr], -1) + 1

    g = Grid(x=X.reshape(n).copy(), y=Y.reshape(n).copy(), nx=np.zeros(n), ny=np.ones(n),
             min_dist=np.zeros(n), flag_1=flag_1.reshape(n), flag_2=flag_2.reshape(n),
             left=left.reshape(n), right=right.reshape(n),
             nbhs=nbhs.reshape(n).astype(np.int32), conn=flat_conn,
             original_id=np.arange(1, n + 1, dtype=np.int32),
             qtdepth=np.zeros(n, dtype=np.int32), shapes=1,
             name=name or f"naca00{int(round(thickness * 100)):02d}_{ni}x{nj}")
    if augment:
        _augment_stencils(g, ni, nj, min_rel_det)
        _repair_stencils(g, ni, nj, min_rel_det)
    # min_dist: distance to the nearest stencil neighbour (the reference reads
    # it from the grid file and never recomputes it)
    kmax = int(g.nbhs.max())
    slot = np.arange(kmax)[:, None] < g.nbhs[None, :]
    idx = np.where(slot, g.conn[:kmax] - 1, 0)
    d = np.hypot(g.x[idx] - g.x[None, :], g.y[idx] - g.y[None, :])
    g.min_dist = np.where(slot, d, np.inf).min(axis=0)
    g.nx, g.ny = reference_normals(g)
    g.validate()
    return g


# Configurations the benchmarks and parity tests use (ni x nj, flow).  C1 uses
# a 5e-3 first spacing: at 160 points around, 1e-3 gives near-wall cells of
# aspect ratio ~20 on which the scheme has a growing wall mode (the oracle
# diverges near iteration 560 at CFL 0.2 and near 1100 at CFL 0.1).  The
# same mode grows at the sharp trailing edge of the fine cosine-spaced grids,
# where straight rays leave the surface at ~7 degrees: C2 and C5 end on a NaN
# residue near iteration 370 (their benchmarks time the first iterations).
# C3 and the batched instances use wall points uniform in arc length with
# square first cells ("arc", "match"), stable over 3000 iterations at
# M 0.63-0.85 up to 640x400.
CONFIGS = {
    "C1": dict(ni=160, nj=100, mach=0.63, aoa=2.0, inner_iterations=0, iters=1000,
               seed=1000, first_spacing=5e-3),
    "C2": dict(ni=1280, nj=800, mach=0.85, aoa=1.0, inner_iterations=3, iters=5000,
               seed=2000, first_spacing=1e-3),
    "C3": dict(ni=640, nj=400, mach=0.63, aoa=2.0, inner_iterations=0, iters=2000,
               seed=3000, first_spacing="match", spacing="arc"),
    "C5": dict(ni=2560, nj=1600, mach=0.8, aoa=1.25, inner_iterations=0, iters=5000,
               seed=5000, first_spacing=1e-3),
    # profiling case: the C2 flow on half the points (working set still > L2)
    "P": dict(ni=1024, nj=512, mach=0.85, aoa=1.0, inner_iterations=3, iters=100,
              seed=9000, first_spacing=1e-3),
}
FLOW_DEFAULTS = dict(cfl=0.2, vl_const=5.0, power=0.0, tscheme="ssprk43")


def config_grid(name: str, **overrides) -> Grid:
    c = dict(CONFIGS[name])
    c.update(overrides)
    return naca_ogrid(c["ni"], c["nj"], seed=c["seed"], first_spacing=c["first_spacing"],
                      spacing=c.get("spacing", "cosine"), name=f"{name}_{c['ni']}x{c['nj']}")


def batch_instances(n_inst: int = 64, config: int = 4, n_min: int = 4000, n_max: int = 256000,
                    aspect: float = 1.6, mach=(0.5, 0.8), aoa=(-2.0, 4.0),
                    thickness=(0.08, 0.16), first_spacing="match", spacing="arc",
                    inner_iterations=0, build: bool = True):
    """Instances of a batched workload: instance k draws from PCG64 seeded
    1000*config + k a point count log-uniform in [n_min, n_max] (ni x nj with
    ni ~ aspect*nj, ni even), a Mach number, an angle of attack and a
    thickness, each uniform in its range.  Returns (grids, flows, specs); with
    build=False the grids are None (only the draws).  The grids are C3's kind
    (arc-length wall spacing, square first cells), free of the growing
    trailing-edge mode (see CONFIGS)."""
    grids, flows, specs = [], [], []
    for k in range(n_inst):
        rng = np.random.default_rng(1000 * config + k)
        n = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        m = float(rng.uniform(*mach))
        a = float(rng.uniform(*aoa))
        t = float(rng.uniform(*thickness))
        nj = max(8, int(round(np.sqrt(n / aspect))))
        ni = max(16, 2 * int(round(aspect * nj / 2)))
        spec = dict(ni=ni, nj=nj, mach=m, aoa=a, thickness=t, seed=1000 * config + k)
        specs.append(spec)
        flow = dict(FLOW_DEFAULTS)
        flow.update(mach=m, aoa=a, inner_iterations=inner_iterations)
        flows.append(flow)
        grids.append(naca_ogrid(ni, nj, thickness=t, seed=spec["seed"], spacing=spacing,
                                first_spacing=first_spacing, name=f"B{config}_{k}_{ni}x{nj}")
                     if build else None)
    return grids, flows, specs


def config_flow(name: str) -> dict:
    """Solver parameters of a configuration (case.in keys)."""
    c = CONFIGS[name]
    f = dict(FLOW_DEFAULTS)
    f.update(mach=c["mach"], aoa=c["aoa"], inner_iterations=c["inner_iterations"])
    return f
