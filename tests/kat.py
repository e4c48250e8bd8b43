"""Known-answer cases taken from the reference's own unit tests.

* EOS6: test/src/unit/natural_core_test.cpp:28-125 -- six-component PR at
  p = 15 MPa, T = 387.45 K; liquid/vapour Z pinned to 2e-12, component
  fugacities to 2e-8 (relative, the test's near() scale).
* FLASH4: test/src/unit/three_phase_flash_test.cpp:62-191 -- CO2/CH4/nC16/H2O
  PR at 50 bar, 350 K, z = (0.75, 0.025, 0.025, 0.20): three phases, closure
  1e-10, material balance 2e-8, fugacity equality 2e-6.
"""
from __future__ import annotations

import math

import numpy as np

from nonenone_b200.abi import EOS_PR, FluidDesc, MAX_NC


def _fluid(tc, pc, vc, om, mw, kij, water, min_comp):
    d = FluidDesc()
    n = len(tc)
    d.nc = n
    d.eos_model = EOS_PR
    d.eos_type = 1
    d.water_component = water
    d.omega_a, d.omega_b = 0.4572355, 0.0779691
    d.m1, d.m2 = 2.414213562373095, -0.414213562373095
    d.minimum_composition = min_comp
    for i in range(n):
        d.tc[i], d.pc[i], d.vc[i], d.acentric[i], d.mw[i] = tc[i], pc[i], vc[i], om[i], mw[i]
        for j in range(n):
            d.kij[i * MAX_NC + j] = kij[i][j]
    return d


def eos6_fluid():
    return _fluid(
        [189.515, 304.2, 387.607, 597.497, 698.515, 875.0],
        [4580011.59, 7386592.50, 4095515.97, 3345244.875, 1768374.5625, 1169006.79],
        [9.97012032965401e-5, 9.26344713533338e-5, 0.000217076707259486,
         0.000381162235869935, 0.000721410148917871, 0.00113570073874421],
        [0.00854, 0.228, 0.16733, 0.38609, 0.80784, 1.23141],
        [0.0161594, 0.04401, 0.0455725, 0.11774, 0.248827, 0.48152],
        [[0.0, 0.00070981, 0.00077754, 0.0100, 0.0110, 0.0110],
         [0.00070981, 0.0, 0.1500, 0.1500, 0.1500, 0.1500],
         [0.00077754, 0.1500, 0.0, 0.0, 0.0, 0.0],
         [0.0100, 0.1500, 0.0, 0.0, 0.0, 0.0],
         [0.0110, 0.1500, 0.0, 0.0, 0.0, 0.0],
         [0.0110, 0.1500, 0.0, 0.0, 0.0, 0.0]],
        -1, 1.0e-8)


EOS6_P = 15.0e6
EOS6_T = 387.45
EOS6_X = np.array([0.3246914, 0.0128351, 0.2278401, 0.2606985, 0.1134144, 0.0605206])
EOS6_Y = np.array([0.808671, 0.025284, 0.1487798, 0.0175878, 0.0006759, 1.51e-06])
EOS6_ZL = 0.66880987807546899
EOS6_ZV = 0.84105046763526459
EOS6_FL = np.array([11148938.7289865, 285739.262764987, 958802.358789237, 32132.229549948,
                    222.962965571357, 0.0303098653818211])
EOS6_FV = np.array([11364784.8024743, 289457.590456904, 964022.546010914, 31595.5016348791,
                    198.090892606485, 0.0143840907404893])


def flash4_fluid():
    return _fluid(
        [304.2, 190.6, 717.0, 647.3],
        [73.8e5, 46.0e5, 14.2e5, 220.5e5],
        [9.4e-5, 9.9e-5, 9.0e-4, 5.6e-5],
        [0.225, 0.008, 0.742, 0.344],
        [0.0440098, 0.016043, 0.22644, 0.01801528],
        [[0.0, 0.1000, 0.1250, 0.1896],
         [0.1000, 0.0, 0.0780, 0.4850],
         [0.1250, 0.0780, 0.0, 0.5000],
         [0.1896, 0.4850, 0.5000, 0.0]],
        3, 1.0e-30)


FLASH4_P = 50.0e5
FLASH4_T = 350.0
FLASH4_Z = np.array([0.75, 0.025, 0.025, 0.20])


def near(actual, expected, tol):
    """The reference tests' near(): |a-e| <= tol * max(1, |a|, |e|)."""
    actual = np.asarray(actual, dtype=float)
    expected = np.asarray(expected, dtype=float)
    scale = np.maximum(1.0, np.maximum(np.abs(actual), np.abs(expected)))
    return np.all(np.abs(actual - expected) <= tol * scale)


def check_flash4(beta, sat, comp, Z, fug_o, fug_g, fug_w, floor=1.0e-30):
    """Invariants of three_phase_flash_test.cpp:128-191 for one result."""
    assert near(beta.sum(), 1.0, 1e-10)
    assert near(sat.sum(), 1.0, 1e-10)
    assert np.all(beta > 0) and np.all(sat > 0) and np.all(Z > 0)
    for p in range(3):
        assert np.all(comp[p] >= 0) and near(comp[p].sum(), 1.0, 1e-10)
    rec = (beta[:, None] * comp).sum(axis=0)
    assert near(rec, FLASH4_Z, 2e-8)
    assert comp[0][3] > 1e-5 and comp[1][3] > 1e-5
    assert comp[2][0] > 1e-6 and comp[2][3] > 0.9
    rel = lambda a, b: abs(a - b) / max(1.0, abs(a), abs(b))
    for c in range(4):
        assert rel(fug_o[c], fug_g[c]) < 2e-6
        if comp[2][c] > 10 * floor:
            assert rel(fug_o[c], fug_w[c]) < 2e-6
