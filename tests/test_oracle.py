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


def test_oracle_cpa_water_methanol_kat(reference):
    """SRK-CPA water/methanol liquid compressibility recorded by the reference
    (case/five_component_eos_tuned_compare/RUN_REPORT.md:105, the water_methanol
    case of test/src/benchmark/cpa_phase_benchmark.cpp): Z = 0.002920191895."""
    from nonenone_b200.abi import CPA_SRK, EOS_CPA, MAX_NC, FluidDesc
    d = FluidDesc()
    d.nc, d.eos_model, d.eos_type, d.water_component = 2, EOS_CPA, 1, 0
    d.omega_a, d.omega_b, d.m1, d.m2, d.minimum_composition = 0.42748, 0.08664, 1.0, 0.0, 1.0e-30
    for i, (tc, pc, vc, om, mw) in enumerate(((647.3, 22.0483e6, 5.60e-5, 0.344, 0.018015),
                                              (512.6, 8.0959e6, 1.18e-4, 0.559, 0.032042))):
        d.tc[i], d.pc[i], d.vc[i], d.acentric[i], d.mw[i] = tc, pc, vc, om, mw
    d.kij[0 * MAX_NC + 1] = d.kij[1 * MAX_NC + 0] = -0.09
    for i, (a0, b, c1, eps, beta, sites) in enumerate(((0.12277, 1.4515e-5, 0.67359, 16655.0, 0.0692, 2),
                                                       (0.40531, 3.0978e-5, 0.43102, 24591.0, 0.0161, 1))):
        d.cpa_a0[i], d.cpa_b[i], d.cpa_c1[i] = a0, b, c1
        d.cpa_epsilon[i], d.cpa_beta[i] = eps, beta
        d.cpa_donor_sites[i] = d.cpa_acceptor_sites[i] = sites
    d.cpa_physical_term = CPA_SRK
    d.cpa_max_association_iterations, d.cpa_association_tolerance, d.cpa_association_damping = 2000, 1e-12, 0.2
    Z, _ = reference.eos_phase_batch(d, [233183.46666657156], [389.375], [[0.185], [0.815]], [0])
    assert abs(Z[0] - 0.002920191895) < 5e-13
