"""Structured-grid connection graph (nonenone_b200.grid) against the reference's
geometry rules: face order, TPFA half transmissibilities in series, the
transmissibility floor, and the gravity term of vertical faces
(grid/include/structuredgrid/structuredgrid.hpp:602-668,876-907,
structured_cartesian_geometry.hpp:19-71)."""
import numpy as np

from nonenone_b200.grid import GRAVITY, MILLIDARCY, StructuredGrid, axis_centers
from nonenone_b200.synth import natural_case


def test_60x20x1_case_counts_and_symmetry():
    grid, P, z = natural_case(0)
    assert grid.ncell == 1200 and grid.nfaces == 2320 and grid.nconn == 4640
    assert P.shape == (1200,) and z.shape == (1200, 3)
    assert np.allclose(z.sum(axis=1), 1.0)
    for c in range(grid.ncell):
        for k in range(grid.conn_offset[c], grid.conn_offset[c + 1]):
            nb = grid.conn_neighbor[k]
            back = [j for j in range(grid.conn_offset[nb], grid.conn_offset[nb + 1])
                    if grid.conn_neighbor[j] == c]
            assert len(back) == 1
            assert grid.conn_trans[back[0]] == grid.conn_trans[k]
    assert not grid.conn_gravity.any()   # one layer: no vertical faces
    assert np.all(grid.volume == 10.0 * 10.0 * 5.0)


def test_face_order_and_transmissibility_formula():
    nx, ny, nz = 4, 3, 3
    dx, dy, dz = 10.0, 20.0, [2.0, 3.0, 5.0]
    n = nx * ny * nz
    rng = np.random.default_rng(3)
    perm = rng.uniform(10, 500, (n, 3)) * MILLIDARCY
    g = StructuredGrid(nx, ny, nz, dx, dy, dz, perm, np.full(n, 0.2))
    c = 1 + nx * (1 + ny * 1)   # interior cell (1, 1, 1)
    nbs = g.conn_neighbor[g.conn_offset[c]:g.conn_offset[c + 1]]
    assert list(nbs) == [c - 1, c + 1, c - nx, c + nx, c - nx * ny, c + nx * ny]
    for k, nb in zip(range(g.conn_offset[c], g.conn_offset[c + 1]), nbs):
        axis = [0, 0, 1, 1, 2, 2][k - g.conn_offset[c]]
        w = {0: (dx, dx), 1: (dy, dy), 2: (dz[g.k[c]], dz[g.k[nb]])}[axis]
        area = {0: (dy * dz[g.k[c]], dy * dz[g.k[nb]]), 1: (dx * dz[g.k[c]], dx * dz[g.k[nb]]),
                2: (dx * dy, dx * dy)}[axis]
        h1 = perm[c, axis] * area[0] / (0.5 * w[0])
        h2 = perm[nb, axis] * area[1] / (0.5 * w[1])
        assert np.isclose(g.conn_trans[k], 1.0 / (1.0 / h1 + 1.0 / h2), rtol=1e-15)
        zc = axis_centers(dz)
        expect_g = (zc[g.k[c]] - zc[g.k[nb]]) * GRAVITY if axis == 2 else 0.0
        assert g.conn_gravity[k] == expect_g


def test_zero_permeability_closes_the_face():
    perm = np.full((2, 3), 100 * MILLIDARCY)
    perm[1, 0] = 0.0
    g = StructuredGrid(2, 1, 1, 5.0, 5.0, 5.0, perm, np.full(2, 0.2))
    assert np.all(g.conn_trans == 0.0)


def test_axis_centers_are_cumulative():
    assert np.allclose(axis_centers([2.0, 3.0, 5.0]), [1.0, 3.5, 7.5])
