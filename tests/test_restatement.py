"""The plain-C restatement (oracle/nz_oracle.c) pinned against the
reference's known answers and against the reference's own code (CPU only)."""
import numpy as np
import pytest

from nonenone_b200 import abi
from nonenone_b200.fluids import make_fluid
from oracle import restatement as rs
from tests import kat

R = 8.31446261815324

pytestmark = pytest.mark.skipif(not rs.available(), reason="oracle restatement not built")


def test_restatement_eos_kat():
    f = kat.eos6_fluid()
    ZL, lL = rs.phase(f, kat.EOS6_P, kat.EOS6_T, kat.EOS6_X, abi.OIL)
    ZV, lV = rs.phase(f, kat.EOS6_P, kat.EOS6_T, kat.EOS6_Y, abi.GAS)
    assert kat.near(ZL, kat.EOS6_ZL, 2e-12) and kat.near(ZV, kat.EOS6_ZV, 2e-12)
    assert kat.near(np.exp(lL) * kat.EOS6_X * kat.EOS6_P, kat.EOS6_FL, 2e-8)
    assert kat.near(np.exp(lV) * kat.EOS6_Y * kat.EOS6_P, kat.EOS6_FV, 2e-8)
    # density and LBC viscosity known answers (natural_core_test.cpp:109-117)
    mw = np.array([f.mw[i] for i in range(6)])
    rhoL = kat.EOS6_P / (R * kat.EOS6_T * ZL)
    rhoV = kat.EOS6_P / (R * kat.EOS6_T * ZV)
    assert kat.near(rhoL * (kat.EOS6_X @ mw), 725.8104330709524, 2e-12)
    assert kat.near(rhoV * (kat.EOS6_Y @ mw), 128.44402682548275, 2e-12)
    assert kat.near(rs.lbc_viscosity(f, kat.EOS6_X, rhoL, kat.EOS6_T), 1.2351230861591054e-4, 3e-12)
    assert kat.near(rs.lbc_viscosity(f, kat.EOS6_Y, rhoV, kat.EOS6_T), 1.8313005681915054e-5, 3e-12)


@pytest.mark.parametrize("eos_model", [abi.EOS_PR, abi.EOS_SW])
def test_restatement_eos_equals_reference(reference, eos_model):
    f = make_fluid(eos_model=eos_model)
    rng = np.random.default_rng(11)
    n = 500
    P, T = rng.uniform(1e6, 60e6, n), rng.uniform(290, 450, n)
    x = rng.dirichlet([1, 1, 1], n).T.copy()
    role = rng.integers(0, 3, n).astype(np.int8)
    sal = rng.uniform(0, 2, n)
    Zr, lr = reference.eos_phase_batch(f, P, T, x, role, salinity=sal)
    for i in range(n):
        Z, l = rs.phase(f, P[i], T[i], x[:, i], role[i], sal[i])
        if not np.isfinite(Zr[i]):
            assert not np.isfinite(Z)
            continue
        assert kat.near(Z, Zr[i], 1e-14) and kat.near(l, lr[:, i], 1e-13)


def test_golden_flash_satisfies_equilibrium(golden):
    """Every converged multiphase point of the committed reference fixture
    satisfies the reference's acceptance test (|d ln f| <= 10 * 1e-9 on
    non-floor components, material balance) under the restated EOS, and
    two-phase points reproduce their phase fraction by Rachford-Rice."""
    g = golden("flash_pr_nc3.npz")
    f = make_fluid()
    checked = 0
    for i in np.where(g["status"] == 0)[0][:400]:
        pres = int(g["presence"][i])
        act = [p for p in range(3) if (pres >> p) & 1]
        x = g["composition"][:, :, i]
        beta = g["beta"][:, i]
        rec = (beta[:, None] * x).sum(axis=0)
        z = g["z"][:, i] / g["z"][:, i].sum()
        assert np.abs(rec - z).max() < 1e-9
        if len(act) < 2:
            continue
        ref_p = act[0]
        _, lr = rs.phase(f, g["P"][i], g["T"][i], x[ref_p], ref_p)
        for p in act[1:]:
            _, lp = rs.phase(f, g["P"][i], g["T"][i], x[p], p)
            m = (x[ref_p] > 1e-29) & (x[p] > 1e-29)
            d = np.abs(np.log(x[ref_p] * np.exp(lr)) - np.log(x[p] * np.exp(lp)))[m]
            assert d.max() <= 1e-8, (i, d.max())
        if len(act) == 2:
            a, b = act
            K = x[b] / x[a]
            ok, bb = rs.rr2(z, K, init=0.5)
            assert ok and abs(bb - beta[b]) < 1e-8
        checked += 1
    assert checked > 100
