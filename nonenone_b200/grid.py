"""Structured Cartesian grid -> the directed connection graph of the Natural assembly.

Restates the reference's structured-grid geometry
(grid/include/structuredgrid/structuredgrid.hpp, structured_cartesian_geometry.hpp):

* global cell index ``i + nx * (j + ny * k)``;
* each cell's faces in the order XMinus, XPlus, YMinus, YPlus, ZMinus, ZPlus
  (gridenums.hpp:42-51), boundary faces skipped;
* half transmissibility ``T_half = K_axis * |A_n| / (0.5 * width_axis)`` with
  ``A_n`` the product of the two other widths (structuredgrid.hpp:876-907,
  structured_cartesian_geometry.hpp:26-58), and ``T = 1 / (1/T1 + 1/T2)``, zero
  when either half is <= 1e-30 (structuredgrid.hpp:642-668);
* gravity term ``(zc[k] - zc[k_nb]) * 9.80665`` for vertical faces, zero
  otherwise, with ``zc`` the cumulative cell centres (k grows downward;
  structuredgrid.hpp:611-624, structured_cartesian_geometry.hpp:60-71);
* cell volume ``dx * dy * dz``.
"""
from __future__ import annotations

import numpy as np

GRAVITY = 9.80665
TRANS_EPS = 1.0e-30
MILLIDARCY = 9.869233e-16


def axis_centers(widths):
    widths = np.asarray(widths, dtype=np.float64)
    centers = np.zeros_like(widths)
    position = 0.0
    for i, w in enumerate(widths):
        centers[i] = position + 0.5 * w
        position += w
    return centers


class StructuredGrid:
    """Cell/connection arrays of an nx*ny*nz grid.

    ``perm`` is ``[ncell, 3]`` (kx, ky, kz in m^2, cell-major in global order);
    ``dx``, ``dy``, ``dz`` are per-axis width arrays (or scalars).
    """

    def __init__(self, nx, ny, nz, dx, dy, dz, perm, porosity):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        n = self.nx * self.ny * self.nz
        self.ncell = n
        self.dx = np.broadcast_to(np.asarray(dx, np.float64), (self.nx,)).copy()
        self.dy = np.broadcast_to(np.asarray(dy, np.float64), (self.ny,)).copy()
        self.dz = np.broadcast_to(np.asarray(dz, np.float64), (self.nz,)).copy()
        self.perm = np.ascontiguousarray(np.asarray(perm, np.float64).reshape(n, 3))
        self.porosity = np.ascontiguousarray(np.asarray(porosity, np.float64).reshape(n))
        if (self.perm < 0).any() or not np.isfinite(self.perm).all():
            raise ValueError("permeability must be finite and non-negative")
        g = np.arange(n)
        self.i = g % self.nx
        self.j = (g // self.nx) % self.ny
        self.k = g // (self.nx * self.ny)
        wx, wy, wz = self.dx[self.i], self.dy[self.j], self.dz[self.k]
        self.volume = np.ascontiguousarray(wx * wy * wz)
        self._build(wx, wy, wz)

    def _half(self, cells, axis, wx, wy, wz):
        widths = (wx[cells], wy[cells], wz[cells])
        if axis == 0:
            normal = widths[1] * widths[2]
        elif axis == 1:
            normal = widths[0] * widths[2]
        else:
            normal = widths[0] * widths[1]
        return self.perm[cells, axis] * np.abs(normal) / (0.5 * widths[axis])

    def _build(self, wx, wy, wz):
        n = self.ncell
        zc = axis_centers(self.dz)
        # direction: (axis, step, valid mask, neighbour)
        dirs = []
        for axis, size, coord, stride in ((0, self.nx, self.i, 1),
                                          (1, self.ny, self.j, self.nx),
                                          (2, self.nz, self.k, self.nx * self.ny)):
            for step in (-1, 1):
                valid = (coord + step >= 0) & (coord + step < size)
                dirs.append((axis, step, valid, np.arange(n) + step * stride))
        counts = np.zeros(n, np.int64)
        for _, _, valid, _ in dirs:
            counts += valid
        offset = np.zeros(n + 1, np.int64)
        np.cumsum(counts, out=offset[1:])
        nconn = int(offset[-1])
        neighbor = np.empty(nconn, np.int64)
        trans = np.empty(nconn, np.float64)
        gravity = np.zeros(nconn, np.float64)
        fill = offset[:-1].copy()
        for axis, step, valid, nb in dirs:
            cells = np.nonzero(valid)[0]
            nbs = nb[cells]
            slots = fill[cells]
            fill[cells] += 1
            h1 = self._half(cells, axis, wx, wy, wz)
            h2 = self._half(nbs, axis, wx, wy, wz)
            with np.errstate(divide="ignore"):
                t = 1.0 / (1.0 / h1 + 1.0 / h2)
            t = np.where((h1 <= TRANS_EPS) | (h2 <= TRANS_EPS), 0.0, t)
            neighbor[slots] = nbs
            trans[slots] = t
            if axis == 2:
                gravity[slots] = (zc[self.k[cells]] - zc[self.k[nbs]]) * GRAVITY
        self.conn_offset = offset
        self.conn_neighbor = neighbor
        self.conn_trans = trans
        self.conn_gravity = gravity
        self.nconn = nconn

    @property
    def nfaces(self) -> int:
        return self.nconn // 2
