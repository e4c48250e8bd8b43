// fluid_dev.cuh -- the device fluid record built from the C ABI's fluid
// description and flash options (host code; no CUDA runtime needed, so host
// builds of the device headers use it too).
#pragma once

#include "../../include/nonenone_b200.h"
#include "eos.cuh"

namespace nz
{
// Default iteration cap of the lane-refill loops (FluidDev::spinLimit).
constexpr long long kDefaultSpinLimit = 1LL << 26;

inline FluidDev makeFluidDev(const nz_fluid_desc &d, const nz_flash_options &o)
{
    FluidDev f{};
    f.nc = d.nc;
    f.eosModel = d.eos_model;
    f.eosType = d.eos_type;
    f.water = d.water_component;
    f.omegaA = d.omega_a;
    f.omegaB = d.omega_b;
    f.m1 = d.m1;
    f.m2 = d.m2;
    f.minComposition = d.minimum_composition;
    for (int i = 0; i < kMaxNc; ++i)
    {
        f.tc[i] = d.tc[i];
        f.pc[i] = d.pc[i];
        f.vc[i] = d.vc[i];
        f.omega[i] = d.acentric[i];
        f.mw[i] = d.mw[i];
        f.swKind[i] = d.sw_bip_kind[i];
        f.swValue[i] = d.sw_bip_value[i];
    }
    for (int k = 0; k < kMaxNc * kMaxNc; ++k)
        f.kij[k] = d.kij[k];
    f.salinity = d.sw_salinity;
    // CPA parameters and the association scheme (cpaWaterOnlyAnalyticFastPathAvailable_,
    // cpaSingleSymmetricAssociatingComponent_, cpaSingleDonorComponent_; cubic_eos.hpp:1305-1354)
    CpaDev &c = f.cpa;
    for (int i = 0; i < kMaxNc; ++i)
    {
        c.a0[i] = d.cpa_a0[i];
        c.b[i] = d.cpa_b[i];
        c.c1[i] = d.cpa_c1[i];
        c.epsilon[i] = d.cpa_epsilon[i];
        c.beta[i] = d.cpa_beta[i];
        c.donor[i] = i < d.nc ? d.cpa_donor_sites[i] : 0;
        c.acceptor[i] = i < d.nc ? d.cpa_acceptor_sites[i] : 0;
    }
    for (int k = 0; k < kMaxNc * kMaxNc; ++k)
    {
        c.crossEpsilon[k] = d.cpa_cross_epsilon[k];
        c.crossBeta[k] = d.cpa_cross_beta[k];
    }
    c.pengRobinson = d.cpa_physical_term == NZ_CPA_PR ? 1 : 0;
    c.carnahanStarling = d.cpa_radial == NZ_CPA_RADIAL_CARNAHAN_STARLING ? 1 : 0;
    c.maxIterations = d.cpa_max_association_iterations;
    c.tolerance = d.cpa_association_tolerance;
    c.damping = d.cpa_association_damping;
    c.symmetric = -1;
    c.singleDonor = -1;
    int associating = -1, donors = 0, donorComponent = -1;
    bool symmetricOk = true;
    for (int i = 0; i < d.nc; ++i)
    {
        const int dn = c.donor[i], ac = c.acceptor[i];
        if (dn > 0)
        {
            ++donors;
            donorComponent = i;
        }
        if (dn == 0 && ac == 0)
            continue;
        if (associating >= 0 || dn <= 0 || dn != ac)
            symmetricOk = false;
        associating = i;
    }
    if (symmetricOk && associating >= 0)
        c.symmetric = associating;
    else if (donors == 1)
        c.singleDonor = donorComponent;
    f.opt.maxIterations = o.maximum_iterations;
    f.opt.maxRr = o.maximum_rachford_rice_iterations;
    f.opt.maxStability = o.maximum_stability_iterations;
    f.opt.stabilitySsi = o.stability_ssi_before_newton;
    f.opt.stabilityNewton = o.maximum_stability_newton;
    f.opt.twoSsi = o.two_phase_ssi_before_newton;
    f.opt.twoNewton = o.maximum_two_phase_newton;
    f.opt.threeSsi = o.three_phase_ssi_before_newton;
    f.opt.threeNewton = o.maximum_three_phase_newton;
    f.opt.fugacityTol = o.fugacity_tolerance;
    f.opt.rrTol = o.rachford_rice_tolerance;
    f.opt.stabilityTol = o.stability_tolerance;
    f.opt.betaTol = o.phase_fraction_tolerance;
    f.opt.coincidentTol = o.coincident_composition_tolerance;
    f.opt.floor = o.composition_floor;
    f.opt.logKLimit = o.log_k_step_limit;
    f.opt.fdStep = o.numerical_jacobian_step;
    f.spinLimit = kDefaultSpinLimit;
    return f;
}
} // namespace nz
