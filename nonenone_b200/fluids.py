"""Fluid descriptions of the benchmark workloads.

Component constants and where each comes from:

* H2O / CO2 / nC10 (nc=3): Tc, Pc, omega and the three BIPs are the synthetic
  set of the benchmark definition (H2O 647.1 K, 22.064 MPa, 0.344; CO2
  304.13 K, 7.377 MPa, 0.225; nC10 617.7 K, 2.11 MPa, 0.49; k = 0.19 / 0.48 /
  0.10).  Molar masses and critical volumes (needed by LBC viscosity) are the
  reference case's (case/h2o_co2_nc10_2d_benchmark/case_config.hpp:53-58).
  nC10 omega is exactly 0.49, so the strict PR78 switch ``omega > 0.49``
  (models/include/natural/thermo/cubic_eos.hpp:606-613) keeps standard PR m.
* C1, nC4 (case/three_eos_3d_compare/case_config.hpp:142-160), nC16
  (case/scw_co2_nc4_nc16_3d_migration/case_config.hpp:46-55), C2, C3
  (tools/example/pr_c2_c3_nc5/main.cpp:32-36).  BIPs not given by a reference
  case are zero.
"""
from __future__ import annotations

import math

from .abi import (CPA_PR, CPA_RADIAL_SIMPLIFIED, EOS_CPA, EOS_PR, EOS_SW, FluidDesc, MAX_NC,
                  SW_BIP_CO2, SW_BIP_HYDROCARBON, SW_BIP_KIJ)

OMEGA_A = 0.4572355
OMEGA_B = 0.0779691
M1 = 1.0 + math.sqrt(2.0)
M2 = 1.0 - math.sqrt(2.0)

# name: (Tc K, Pc Pa, Vc m3/mol, omega, Mw kg/mol)
COMPONENTS = {
    "H2O": (647.1, 22.064e6, 5.5948e-5, 0.344, 0.018015268),
    "CO2": (304.13, 7.377e6, 9.4118e-5, 0.225, 0.0440098),
    "nC10": (617.7, 2.11e6, 6.10e-4, 0.49, 0.14228168),
    "C1": (190.564002651, 4.599200474e6, 9.862771707e-5, 0.01142, 0.0160428),
    "C2": (305.32, 4.872e6, 1.458e-4, 0.099, 0.03007),
    "C3": (369.83, 4.248e6, 2.000e-4, 0.152, 0.04410),
    "nC4": (425.125, 3.796000017e6, 2.549219298e-4, 0.200810094644, 0.0581222),
    "nC16": (723.0, 1.410e6, 9.0e-4, 0.742, 0.2264412),
}

# Symmetric pair BIPs; unlisted pairs are zero.
PAIR_BIPS = {
    frozenset(("H2O", "CO2")): 0.19,
    frozenset(("H2O", "nC10")): 0.48,
    frozenset(("CO2", "nC10")): 0.10,
    frozenset(("H2O", "C1")): 0.4850,
    frozenset(("H2O", "C2")): 0.5000,
    frozenset(("H2O", "nC4")): 0.5000,
    frozenset(("H2O", "nC16")): 0.5000,
    frozenset(("CO2", "C1")): 0.1000,
    frozenset(("CO2", "C2")): 0.1300,
    frozenset(("CO2", "nC4")): 0.1277,
    frozenset(("CO2", "nC16")): 0.0900,
    frozenset(("C1", "nC4")): 0.09281,
}

H2O_CO2_NC10 = ("H2O", "CO2", "nC10")
SIX_COMPONENT = ("H2O", "CO2", "C1", "nC4", "nC10", "nC16")


def make_fluid(names=H2O_CO2_NC10, eos_model: int = EOS_PR, eos_type: int = 1,
               salinity: float = 0.0) -> FluidDesc:
    """Build an nz_fluid_desc.  H2O must be present; it is the water component."""
    nc = len(names)
    if not 2 <= nc <= MAX_NC:
        raise ValueError("nc must be in 2..8")
    d = FluidDesc()
    d.nc = nc
    d.eos_model = eos_model
    d.eos_type = eos_type
    d.water_component = names.index("H2O") if "H2O" in names else -1
    d.omega_a, d.omega_b, d.m1, d.m2 = OMEGA_A, OMEGA_B, M1, M2
    d.minimum_composition = 1.0e-8
    for i, n in enumerate(names):
        tc, pc, vc, om, mw = COMPONENTS[n]
        d.tc[i], d.pc[i], d.vc[i], d.acentric[i], d.mw[i] = tc, pc, vc, om, mw
        for j, m in enumerate(names):
            if i != j:
                d.kij[i * MAX_NC + j] = PAIR_BIPS.get(frozenset((n, m)), 0.0)
    d.sw_salinity = salinity
    for i, n in enumerate(names):
        if eos_model == EOS_SW and n != "H2O":
            # Aqueous BIP correlations of the SW model (soreide_whitson.hpp:54-134)
            d.sw_bip_kind[i] = SW_BIP_CO2 if n == "CO2" else SW_BIP_HYDROCARBON
        else:
            d.sw_bip_kind[i] = SW_BIP_KIJ
    return d


GAS_CONSTANT = 8.31446261815324

# Standard 4C water of SRK-CPA (models/include/natural/thermo/cubic_plus_association.hpp:31-40)
WATER_4C = dict(a0=0.12277, b=1.4515e-5, c1=0.67359, epsilon=16655.0, beta=0.0692, donor=2, acceptor=2)


def set_cpa(d: FluidDesc, names, physical_term: int = CPA_PR, water: dict | None = None,
            radial: int = CPA_RADIAL_SIMPLIFIED) -> FluidDesc:
    """Make `d` a CPA fluid with the reference factory's defaults
    (case/include/case/fluid_factory.hpp:323-396): every component's cubic part
    from Tc, Pc, omega (PR or SRK form; PR78 c1 for omega > 0.49 when eos_type is
    5), water replaced by the 4C parameter set (or `water`)."""
    R = GAS_CONSTANT
    d.eos_model = EOS_CPA
    d.cpa_physical_term = physical_term
    d.cpa_radial = radial
    d.cpa_max_association_iterations = 2000
    d.cpa_association_tolerance = 1.0e-12
    d.cpa_association_damping = 0.2
    for i, n in enumerate(names):
        tc, pc, _, om, _ = COMPONENTS[n]
        if physical_term == CPA_PR:
            d.cpa_a0[i] = 0.45724 * R * R * tc * tc / pc
            d.cpa_b[i] = 0.07780 * R * tc / pc
            d.cpa_c1[i] = 0.37464 + 1.54226 * om - 0.26992 * om * om
            if d.eos_type == 5 and om > 0.49:
                d.cpa_c1[i] = 0.379642 + 1.48503 * om - 0.164423 * om * om + 0.016666 * om * om * om
        else:
            d.cpa_a0[i] = 0.42748 * R * R * tc * tc / pc
            d.cpa_b[i] = 0.08664 * R * tc / pc
            d.cpa_c1[i] = 0.480 + 1.574 * om - 0.176 * om * om
    if "H2O" in names:
        w = names.index("H2O")
        p = WATER_4C if water is None else water
        d.cpa_a0[w], d.cpa_b[w], d.cpa_c1[w] = p["a0"], p["b"], p["c1"]
        d.cpa_epsilon[w], d.cpa_beta[w] = p["epsilon"], p["beta"]
        d.cpa_donor_sites[w], d.cpa_acceptor_sites[w] = p["donor"], p["acceptor"]
    return d


def make_cpa_h2o_co2_nc10(co2_acceptor: bool = True) -> FluidDesc:
    """The PR-CPA H2O/CO2/nC10 fluid of the reference's 60x20 case
    (case/h2o_co2_nc10_2d_benchmark/case_config.hpp:106-142): water
    a0 = 0.15782, b = 1.4788e-5, c1 = 0.6736, epsilon = 16123 J/mol,
    beta = 0.069662 with two donor and two acceptor sites; CO2 one acceptor site
    cross-associating with water (epsilon 8061.5, beta 0.15182); PR78 c1 for nC10;
    the case's CPA BIPs (H2O-CO2 0.10566, CO2-nC10 0.1141).  Tc, Pc, omega are the
    benchmark set of this module.  `co2_acceptor=False` leaves water the only
    associating component (the analytic site-fraction path)."""
    names = H2O_CO2_NC10
    d = make_fluid(names, eos_type=5)
    for i in range(MAX_NC * MAX_NC):
        d.kij[i] = 0.0
    for (a, b), k in (((0, 1), 0.10566), ((1, 2), 0.1141)):
        d.kij[a * MAX_NC + b] = d.kij[b * MAX_NC + a] = k
    set_cpa(d, names, CPA_PR, water=dict(a0=0.15782, b=1.4788e-5, c1=0.6736, epsilon=16123.0,
                                         beta=0.069662, donor=2, acceptor=2))
    tc, pc, _, om, _ = COMPONENTS["nC10"]
    d.cpa_c1[2] = 0.379642 + 1.48503 * om - 0.164423 * om * om + 0.016666 * om * om * om
    if co2_acceptor:
        d.cpa_epsilon[1], d.cpa_beta[1] = 8061.5, 0.15182
        d.cpa_acceptor_sites[1] = 1
        d.cpa_cross_epsilon[0 * MAX_NC + 1] = 8061.5
        d.cpa_cross_beta[0 * MAX_NC + 1] = 0.15182
    return d


# Component sets of the multi-model and serving workloads, by component count:
# the six-component benchmark set, reduced or extended with C2 / C3.
MODEL_COMPONENTS = {
    3: H2O_CO2_NC10,
    4: ("H2O", "CO2", "C1", "nC10"),
    5: ("H2O", "CO2", "C1", "nC4", "nC10"),
    6: SIX_COMPONENT,
    8: ("H2O", "CO2", "C1", "C2", "C3", "nC4", "nC10", "nC16"),
}


def model_fluid(nc: int, eos: str) -> FluidDesc:
    """The fluid of one model of the multi-model / serving workloads: the
    MODEL_COMPONENTS set of `nc` with eos "pr", "sw" (salinity 1 mol/kg) or
    "cpa" (PR-CPA, 4C water with CO2 as a cross-associating acceptor)."""
    names = MODEL_COMPONENTS[nc]
    if eos == "pr":
        return make_fluid(names)
    if eos == "sw":
        return make_fluid(names, eos_model=EOS_SW, salinity=1.0)
    if eos == "cpa":
        return make_cpa_names(names)
    raise ValueError(f"unknown eos {eos!r}")


def make_cpa_six() -> FluidDesc:
    """The six-component PR-CPA fluid of the 200x200x50 benchmark grid:
    {H2O, CO2, C1, nC4, nC10, nC16} with the critical data and BIPs of
    make_fluid(SIX_COMPONENT), water self-associating with the 4C parameters
    of make_cpa_h2o_co2_nc10 and CO2 a cross-associating acceptor (the
    single-donor association path), PR physical term."""
    return make_cpa_names(SIX_COMPONENT)


def make_cpa_names(names) -> FluidDesc:
    """PR-CPA on a component set holding H2O and CO2 (see make_cpa_six)."""
    d = make_fluid(names, eos_type=5)
    set_cpa(d, names, CPA_PR, water=dict(a0=0.15782, b=1.4788e-5, c1=0.6736, epsilon=16123.0,
                                         beta=0.069662, donor=2, acceptor=2))
    co2 = names.index("CO2")
    w = names.index("H2O")
    d.cpa_epsilon[co2], d.cpa_beta[co2] = 8061.5, 0.15182
    d.cpa_acceptor_sites[co2] = 1
    d.cpa_cross_epsilon[w * MAX_NC + co2] = 8061.5
    d.cpa_cross_beta[w * MAX_NC + co2] = 0.15182
    return d
