"""CPU tests of the synthetic grid generator."""
import numpy as np
import pytest

from mfcfd_b200.grid import (INTERIOR, OUTER, WALL, config_grid, naca_ogrid, reference_normals,
                             split_conditioning)


def test_deterministic_from_seed():
    a = naca_ogrid(40, 16, seed=9)
    b = naca_ogrid(40, 16, seed=9)
    c = naca_ogrid(40, 16, seed=10)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.conn, b.conn)
    assert not np.array_equal(a.x, c.x)


def test_layout_and_ranges():
    g = naca_ogrid(40, 16, seed=1)
    g.validate()
    assert g.n == 640
    assert (g.flag_1[:40] == WALL).all() and (g.flag_1[-40:] == OUTER).all()
    assert (g.flag_2[:40] == 1).all() and (g.flag_2[40:] == 0).all()
    assert (g.nbhs[g.flag_1 == INTERIOR] >= 8).all()
    assert (g.nbhs[g.flag_1 != INTERIOR] >= 5).all()
    assert np.array_equal(g.original_id, np.arange(1, 641))
    # outer ring is the circle of radius 20 about (0.5, 0)
    r = np.hypot(g.x[-40:] - 0.5, g.y[-40:])
    assert np.allclose(r, 20.0)


def test_normals_point_out_of_body_and_domain():
    g = naca_ogrid(64, 20, seed=2)
    nx, ny = reference_normals(g)
    wall = g.flag_1 == WALL
    outer = g.flag_1 == OUTER
    # wall normals point away from the chord line, outer ones away from the centre
    assert np.all((g.x[wall] - 0.5) * nx[wall] + g.y[wall] * ny[wall] > 0)
    assert np.all((g.x[outer] - 0.5) * nx[outer] + g.y[outer] * ny[outer] > 0)


@pytest.mark.parametrize("ni,nj", [(160, 100), (640, 400)])
def test_split_lists_well_posed(ni, nj):
    g = naca_ogrid(ni, nj, seed=3, first_spacing=1e-3 if ni > 160 else 5e-3)
    rel, cnt = split_conditioning(g)
    assert rel.min() >= 1e-4
    used = np.isfinite(rel)
    assert (cnt[used] >= 2).all()


def test_split_lists_well_posed_at_fine_trailing_edge():
    # 2560 cosine-spaced wall points with a 1e-3 first spacing (the C5 wall
    # and spacing): nearest-first augmentation leaves trailing-edge wall
    # points with a list of collinear wall points; the repair pass rebuilds
    # them within MAX_NBHS
    g = naca_ogrid(2560, 16, seed=5000, first_spacing=1e-3)
    rel, cnt = split_conditioning(g)
    assert rel.min() >= 1e-4
    assert (cnt[np.isfinite(rel)] >= 2).all()
    assert int(g.nbhs.max()) <= 20


def test_config_c1_size():
    g = config_grid("C1")
    assert g.n == 16000
    assert 7.9 < g.mean_nbhs() < 8.0


def test_repair_leaves_well_posed_grids_unchanged():
    # the repair pass only rebuilds points the first pass left singular: a
    # grid without such points (the 160x100 C1 wall) is the same with and
    # without it
    from mfcfd_b200 import grid as G
    full = config_grid("C1")
    ni, nj = 160, 100
    first = naca_ogrid(ni, nj, seed=1000, first_spacing=5e-3, augment=False)
    G._augment_stencils(first, ni, nj, 1e-4)
    assert G._repair_stencils(first, ni, nj, 1e-4) == 0
    assert np.array_equal(first.conn, full.conn) and np.array_equal(first.nbhs, full.nbhs)
