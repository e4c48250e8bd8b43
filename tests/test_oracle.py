"""The oracle pinned against the reference's own known answers (CPU only)."""
import numpy as np
import pytest

from nonenone_b200 import abi
from nonenone_b200.fluids import make_fluid
from tests import kat


def _fugacity(P, x, lnphi):
    return np.exp(lnphi) * x * P


def test_reference_eos_matches_natural_core_kat(reference):
    f = kat.eos6_fluid()
    P = np.full(2, kat.EOS6_P)
    T = np.full(2, kat.EOS6_T)
    x = np.stack([kat.EOS6_X, kat.EOS6_Y], axis=1)
    Z, lnphi = reference.eos_phase_batch(f, P, T, x, [abi.OIL, abi.GAS])
    assert kat.near(Z[0], kat.EOS6_ZL, 2e-12)
    assert kat.near(Z[1], kat.EOS6_ZV, 2e-12)
    assert kat.near(_fugacity(kat.EOS6_P, kat.EOS6_X, lnphi[:, 0]), kat.EOS6_FL, 2e-8)
    assert kat.near(_fugacity(kat.EOS6_P, kat.EOS6_Y, lnphi[:, 1]), kat.EOS6_FV, 2e-8)


def test_reference_flash_three_phase_kat(reference):
    f = kat.flash4_fluid()
    out = reference.flash_batch(f, [kat.FLASH4_P], [kat.FLASH4_T], kat.FLASH4_Z.reshape(4, 1))
    assert out["status"][0] == abi.FLASH_CONVERGED and out["presence"][0] == 7
    comp = out["composition"][:, :, 0]
    P = np.full(3, kat.FLASH4_P)
    T = np.full(3, kat.FLASH4_T)
    Z, lnphi = reference.eos_phase_batch(f, P, T, comp.T.copy(), [abi.OIL, abi.GAS, abi.WATER])
    fug = [_fugacity(kat.FLASH4_P, comp[p], lnphi[:, p]) for p in range(3)]
    kat.check_flash4(out["beta"][:, 0], out["saturation"][:, 0], comp, Z, *fug)


@pytest.mark.parametrize("name", ["flash_pr_nc3.npz", "flash_sw_nc3.npz", "flash_pr_nc6.npz"])
def test_golden_fixtures_are_the_reference(reference, golden, name):
    """The committed fixtures are exactly what the reference computes now."""
    g = golden(name)
    from nonenone_b200.fluids import SIX_COMPONENT
    fluid = {"flash_pr_nc3.npz": make_fluid(),
             "flash_sw_nc3.npz": make_fluid(eos_model=abi.EOS_SW),
             "flash_pr_nc6.npz": make_fluid(SIX_COMPONENT)}[name]
    idx = np.arange(0, g["P"].shape[0], 7)
    out = reference.flash_batch(fluid, g["P"][idx], g["T"][idx], g["z"][:, idx],
                                salinity=None if "salinity" not in g else g["salinity"][idx])
    for k in ("status", "presence", "beta", "composition", "saturation"):
        assert np.array_equal(out[k], g[k][..., idx]), k


def test_golden_label_mix(golden):
    """The batched-flash mixture is roughly 40/40/20 single/two/three-phase."""
    g = golden("flash_pr_nc3.npz")
    pres = g["presence"][g["status"] == 0]
    n = pres.size
    single = np.isin(pres, [1, 2, 4]).sum() / n
    three = (pres == 7).sum() / n
    assert 0.33 < single < 0.47 and 0.14 < three < 0.26
