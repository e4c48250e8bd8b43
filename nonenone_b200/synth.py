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


def raw_box_points(n: int, seed: int = 12345):
    """The unresampled box: P ~ U[5,40] MPa, T ~ U[303,423] K, z ~ Dir(2,1,1)."""
    rng = np.random.default_rng(seed)
    P = rng.uniform(5e6, 40e6, n)
    T = rng.uniform(303.0, 423.0, n)
    z = np.ascontiguousarray(rng.dirichlet([2.0, 1.0, 1.0], n).T)
    return P, T, z
