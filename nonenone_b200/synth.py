"""Seeded synthetic inputs with the shapes of the benchmark workloads.

Batched P-T-z flash (1,048,576 points, nc=3 H2O/CO2/nC10):
  P ~ U[5,40] MPa, T ~ U[303,423] K, z ~ Dirichlet(2,1,1) is the raw box.  The
  raw box is ~0.05 % single-phase, ~89 % two-phase, ~10.5 % three-phase by the
  reference label, so points are drawn from a label-free proposal mixture
  calibrated once against the reference flash (20k-point samples):
    45 % "dry"   z_H2O ~ U[0,5e-4], (CO2,nC10) ~ Dir(1,1)      -> 87.5 % 1-ph
    32 % "box"   the raw box                                  -> 88 % 2-ph
    23 % "3ph"   P ~ U[5,12] MPa, T ~ U[340,423] K, z ~ Dir(2,2,0.6) -> 73 % 3-ph
  which gives roughly 40 % / 40 % / 20 % single / two / three-phase.
  Soreide-Whitson points add salinity ~ U[0,2] mol/kg.
  benchmark_points adds the 5 % slice of points next to a phase boundary
  (boundary_points: P bisected to a label change, then offset by <= 5e-6
  relative).
"""
from __future__ import annotations

import numpy as np

MIX = (("dry", 0.45), ("box", 0.32), ("3ph", 0.23))


def flash_points(n: int, seed: int = 1, salinity: bool = False):
    """Return P[n], T[n], z[3, n] (and salinity[n] when asked) as float64."""
    rng = np.random.default_rng(seed)
    counts = [int(round(w * n)) for _, w in MIX]
    counts[-1] = n - sum(counts[:-1])
    P, T, Z = [], [], []
    for (kind, _), m in zip(MIX, counts):
        if kind == "dry":
            zw = rng.uniform(0.0, 5.0e-4, m)
            r = rng.dirichlet([1.0, 1.0], m)
            z = np.stack([zw, (1 - zw) * r[:, 0], (1 - zw) * r[:, 1]])
            p = rng.uniform(5e6, 40e6, m)
            t = rng.uniform(303.0, 423.0, m)
        elif kind == "box":
            z = rng.dirichlet([2.0, 1.0, 1.0], m).T
            p = rng.uniform(5e6, 40e6, m)
            t = rng.uniform(303.0, 423.0, m)
        else:
            z = rng.dirichlet([2.0, 2.0, 0.6], m).T
            p = rng.uniform(5e6, 12e6, m)
            t = rng.uniform(340.0, 423.0, m)
        P.append(p)
        T.append(t)
        Z.append(z)
    P = np.concatenate(P)
    T = np.concatenate(T)
    Z = np.concatenate(Z, axis=1)
    perm = rng.permutation(n)
    P, T, Z = P[perm], T[perm], np.ascontiguousarray(Z[:, perm])
    if salinity:
        return P, T, Z, rng.uniform(0.0, 2.0, n)
    return P, T, Z


BOUNDARY_FRACTION = 0.05


def boundary_points(n: int, labels, seed: int = 7, salinity: bool = False, offset=(1.0e-10, 5.0e-6),
                    bisections: int = 44):
    """n points next to a phase boundary (the benchmark's "5 % within
    |TPD| < 1e-6" slice): for (T, z) drawn from the raw box, P is bisected
    between 5 and 40 MPa on a change of the phase label, then moved off the
    boundary by a relative offset of either sign and log-uniform magnitude in
    `offset` (for the H2O/CO2/nC10 fluid the |TPD| of the boundary phase then
    lies between ~1e-12 and ~1e-6, a fraction of the points below 1e-8).

    `labels(P, T, z, salinity)` returns the phase-presence labels of a batch
    (any flash: the oracle when fixtures are made, the GPU flash when the
    benchmark builds its batch; 0 = not converged).  (T, z) pairs whose label
    does not change between 5 and 40 MPa, or whose bracket meets a flash that
    fails, are redrawn: the boundary sought is between two answered phase
    sets, not the edge of the flash's convergence region.  Returns P, T,
    z[3, n] (and salinity)."""
    rng = np.random.default_rng(seed)
    Ps, Ts, Zs, Ss = [], [], [], []
    have = 0
    while have < n:
        m = max(2 * (n - have), 64)
        T = rng.uniform(303.0, 423.0, m)
        z = np.ascontiguousarray(rng.dirichlet([2.0, 1.0, 1.0], m).T)
        sal = rng.uniform(0.0, 2.0, m) if salinity else None
        lo = np.full(m, 5.0e6)
        hi = np.full(m, 40.0e6)
        lab_lo = labels(lo, T, z, sal)
        lab_hi = labels(hi, T, z, sal)
        keep = (lab_lo != lab_hi) & (lab_lo != 0) & (lab_hi != 0)
        lo, hi, T, z, lab_lo = lo[keep], hi[keep], T[keep], np.ascontiguousarray(z[:, keep]), lab_lo[keep]
        sal = None if sal is None else sal[keep]
        answered = np.ones(lo.size, bool)
        for _ in range(bisections):
            mid = 0.5 * (lo + hi)
            lab = labels(mid, T, z, sal)
            answered &= lab != 0
            same = lab == lab_lo
            lo = np.where(same, mid, lo)
            hi = np.where(same, hi, mid)
        mag = 10.0 ** rng.uniform(np.log10(offset[0]), np.log10(offset[1]), lo.size)
        P = 0.5 * (lo + hi) * (1.0 + np.where(rng.uniform(size=lo.size) < 0.5, -mag, mag))
        P, T, z = P[answered], T[answered], np.ascontiguousarray(z[:, answered])
        sal = None if sal is None else sal[answered]
        take = min(P.size, n - have)
        Ps.append(P[:take])
        Ts.append(T[:take])
        Zs.append(z[:, :take])
        if sal is not None:
            Ss.append(sal[:take])
        have += take
    P, T, Z = np.concatenate(Ps), np.concatenate(Ts), np.ascontiguousarray(np.concatenate(Zs, axis=1))
    if salinity:
        return P, T, Z, np.concatenate(Ss)
    return P, T, Z


def benchmark_points(n: int, boundary, seed: int = 1):
    """The batched-flash benchmark's batch: the label mixture of flash_points
    for n - len(boundary) points and the given near-boundary slice
    (boundary_points output, ~5 %) for the rest, shuffled together."""
    nb = boundary[0].shape[0]
    mix = flash_points(n - nb, seed=seed)
    perm = np.random.default_rng(seed + 104729).permutation(n)
    return tuple(np.ascontiguousarray(np.concatenate([a, b], axis=a.ndim - 1)[..., perm])
                 for a, b in zip(mix, boundary))


def raw_box_points(n: int, seed: int = 12345):
    """The unresampled box: P ~ U[5,40] MPa, T ~ U[303,423] K, z ~ Dir(2,1,1)."""
    rng = np.random.default_rng(seed)
    P = rng.uniform(5e6, 40e6, n)
    T = rng.uniform(303.0, 423.0, n)
    z = np.ascontiguousarray(rng.dirichlet([2.0, 1.0, 1.0], n).T)
    return P, T, z


def natural_case(seed: int = 0, nx: int = 60, ny: int = 20, nz: int = 1,
                 dx: float = 10.0, dy: float = 10.0, dz: float = 5.0,
                 perm_median_md: float = 100.0, perm_sigma_ln: float = 1.0,
                 kv_kh: float = 1.0, porosity=(0.15, 0.25), pressure=(10e6, 30e6),
                 alpha=(2.0, 1.0, 1.0)):
    """One Newton evaluation's inputs on a structured grid.

    Defaults are the 60x20x1 H2O/CO2/nC10 case: 10 m x 10 m x 5 m cells,
    permeability lognormal (median 100 mD, sigma_ln 1), porosity U[0.15, 0.25],
    P ~ U[10, 30] MPa, z ~ Dirichlet(2, 1, 1).  Returns (grid, P[ncell],
    z[ncell, nc]).
    """
    from .grid import MILLIDARCY, StructuredGrid
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    kh = perm_median_md * MILLIDARCY * np.exp(perm_sigma_ln * rng.standard_normal(n))
    perm = np.stack([kh, kh, kh * kv_kh], axis=1)
    phi = rng.uniform(porosity[0], porosity[1], n)
    grid = StructuredGrid(nx, ny, nz, dx, dy, dz, perm, phi)
    P = rng.uniform(pressure[0], pressure[1], n)
    z = rng.dirichlet(list(alpha), n)
    return grid, P, np.ascontiguousarray(z)


def natural_case_hydrostatic(seed: int = 3, nx: int = 200, ny: int = 200, nz: int = 50,
                             dx: float = 10.0, dy: float = 10.0, dz: float = 2.0,
                             perm_median_md: float = 50.0, perm_sigma_ln: float = 1.5, kv_kh: float = 0.1,
                             porosity=(0.05, 0.30), p_top: float = 20.0e6, p_gradient: float = 0.01e6,
                             alpha=(4.0, 2.0, 1.0, 1.0, 1.0, 1.0)):
    """The 3-D benchmark grid: nx x ny x nz cells of dx x dy x dz m (200 x 200
    x 50 of 10 x 10 x 2 m: 2,000,000 cells, 5.94 M faces), permeability
    lognormal (median 50 mD, sigma_ln 1.5, kv/kh 0.1), porosity U[0.05, 0.30],
    hydrostatic pressure p_top + p_gradient x depth of the cell centre (20 MPa
    + 0.01 MPa/m), z ~ Dirichlet(alpha).  Returns (grid, P[ncell], z[ncell, nc],
    depth[ncell])."""
    from .grid import MILLIDARCY, StructuredGrid, axis_centers
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    kh = perm_median_md * MILLIDARCY * np.exp(perm_sigma_ln * rng.standard_normal(n))
    perm = np.stack([kh, kh, kh * kv_kh], axis=1)
    phi = rng.uniform(porosity[0], porosity[1], n)
    grid = StructuredGrid(nx, ny, nz, dx, dy, dz, perm, phi)
    depth = axis_centers(np.full(nz, float(dz)))[grid.k]
    P = p_top + p_gradient * depth
    z = rng.dirichlet(list(alpha), n)
    return grid, P, np.ascontiguousarray(z), depth


# Quadratic relative permeabilities of the reference's H2O-CO2-nC10 case
# (case/h2o_co2_nc10_2d_benchmark/benchmark_common.hpp:97-126).
RELPERM_H2O_CO2_NC10 = dict(swc=0.10, sorw=0.15, sgc=0.02, sorg=0.10,
                            krw_max=0.30, krg_max=0.80, kro_max=0.80)


def perturb_natural_state(primary, phase_state, nc: int, seed: int, scale: float = 1.0,
                          remove_fraction: float = 0.1):
    """A Newton iterate near an accepted Natural state (cell-major numpy arrays):
    pressure, phase compositions and saturations jittered, and on
    ``remove_fraction`` of the cells one present phase pushed to a saturation
    of 5e-5 (below the 1e-4 active-set boundary) so that it is removed."""
    rng = np.random.default_rng(seed)
    p = np.array(primary, dtype=np.float64, copy=True)
    n = p.shape[0]
    p[:, 0] *= 1.0 + 0.02 * scale * rng.standard_normal(n)
    ncomp = 3 * (nc - 1)
    p[:, 1:1 + ncomp] += 0.01 * scale * rng.standard_normal((n, ncomp))
    p[:, 1 + ncomp:] += 0.05 * scale * rng.standard_normal((n, 3))
    flags = np.rint(np.asarray(phase_state)[:, 0]).astype(np.int64)
    pick = np.where(rng.uniform(size=n) < remove_fraction)[0]
    for c in pick:
        present = [ph for ph in range(3) if (flags[c] >> ph) & 1]
        ph = present[rng.integers(len(present))]
        p[c, 1 + ncomp + ph] = 5.0e-5
    return p


# Component counts and EOS families of the multi-model workload.
MODEL_NCS = (3, 4, 5, 6, 8)
MODEL_EOS = ("pr", "sw", "cpa")


def model_batch_specs(nmodels: int, cells=(1.0e4, 5.0e5), seed: int = 21, eos=MODEL_EOS, eos_weights=None):
    """The uneven multi-model workload: per model a cell count log-uniform on
    `cells`, a component count uniform over MODEL_NCS and an EOS drawn from
    `eos` (uniform, or with `eos_weights`).  Returns [(nc, eos, cells)]."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(cells[0]), np.log(cells[1])
    n = np.exp(rng.uniform(lo, hi, nmodels)).astype(np.int64)
    ncs = rng.choice(MODEL_NCS, nmodels)
    kinds = rng.choice(len(eos), nmodels, p=eos_weights)
    return [(int(c), eos[int(e)], int(m)) for c, e, m in zip(ncs, kinds, n)]


def model_points(nc: int, n: int, seed: int, depth=(0.0, 250.0), p_top: float = 20.0e6,
                 p_gradient: float = 0.01e6, t_top: float = 373.15, t_gradient: float = 0.03,
                 salinity=(0.0, 2.0)):
    """P, T, z of one model drawn as on the hydrostatic benchmark grid: a depth
    uniform on `depth` m, P = 20 MPa + 0.01 MPa/m and T = 373.15 K + 0.03 K/m
    of it, z ~ Dirichlet(4, 2, 1, ..., 1) over the model's nc components, and a
    salinity U[0, 2] mol/kg (read by Soreide-Whitson models only).
    Returns P[n], T[n], z[nc, n], salinity[n]."""
    rng = np.random.default_rng(seed)
    d = rng.uniform(depth[0], depth[1], n)
    P = p_top + p_gradient * d
    T = t_top + t_gradient * d
    alpha = [4.0, 2.0] + [1.0] * (nc - 2)
    z = np.ascontiguousarray(rng.dirichlet(alpha, n).T)
    sal = rng.uniform(salinity[0], salinity[1], n)
    return P, T, z, sal
