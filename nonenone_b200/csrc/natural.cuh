// natural.cuh -- Natural-formulation cell physics on the device.
//
// Restates, templated on the scalar (double for values, Dual for one
// Jacobian direction per lane):
//   CellStateCodec::decode          state/state_codec.hpp (dependent last
//                                   component, 1e-13 cancellation snap)
//   CellPropertyEvaluator::evaluateFullyCompositional_
//                                   state/cell_property_evaluator.hpp:236-393
//   FluidSystem::eosFlowProperties  fluid_system.hpp:99-125
//   LBC viscosity                   properties/compositional_properties.hpp:106-150
//   computeFluidComponentAccumulation  physics/accumulation.hpp:30-78
//   assembleCellLocalResidual       assembly/cell_residual.hpp:73-425
//   computeFaceMassFlux(Value)      physics/face_flux.hpp:65-430
// with the relative permeabilities of the reference's H2O-CO2-nC10 case
// (case/h2o_co2_nc10_2d_benchmark/benchmark_common.hpp:97-126).
#pragma once

#include "dual.cuh"
#include "cpa.cuh"

namespace nz
{

// Constants of one Natural problem (kernel parameter).
struct NatConst
{
    double temperature;
    double timeStep;
    double fugacityScaling;
    double swc, sorw, sgc, sorg, krwMax, krgMax, kroMax;
    double lbcMwSqrt[kMaxNc];   // initializeLbcConstants_ (compositional_properties.hpp:155-172)
    double lbcEps[kMaxNc];
};

constexpr double kPsi = 0.45359237 * 9.80665 / (0.0254 * 0.0254);   // common/units.hpp
constexpr double kCentipoise = 1.0e-2 * 0.1;
constexpr double kKelvinPerRankine = 5.0 / 9.0;
constexpr double kTraceComposition = 1.0e-14;       // NaturalNumerics::phaseEquilibriumTraceComposition
constexpr double kCancellationBoundary = 1.0e-13;   // NaturalNumerics::dependentCompositionCancellationBoundary

// Device view of one Natural problem.
struct NatGeom
{
    int64_t ncell;
    const double *porosity;
    const double *volume;
    const int64_t *offset;     // [ncell+1] directed connections
    const int64_t *neighbor;   // [nconn]
    const double *trans;       // [nconn]
    const double *gravity;     // [nconn]
    const int64_t *selfSlot;   // [ncell] block index of (c, c)
    const int64_t *connSlot;   // [nconn] block index of (neighbor, c)
    const double *prevAcc;     // [ncell][NC] accumulation of the accepted state
    double *cache;             // [fields][ncell] frozen exterior values
    int columnOrder;           // Jacobian output: 0 pattern (block-row) order, 1 cell-column order
};

// Block index of a Jacobian block in the output array.  Pattern order: the
// BAIJ slot of (c, c) / (neighbor, c).  Cell-column order: cell c's column
// -- its self block, then the block of each connection in connection order --
// is one contiguous run of 1 + nconn(c) blocks starting at c + offset[c].
NZ_BOTH int64_t selfBlock(const NatGeom &g, int64_t c)
{
    return g.columnOrder ? c + g.offset[c] : g.selfSlot[c];
}
NZ_BOTH int64_t connBlock(const NatGeom &g, int64_t c, int64_t j)
{
    return g.columnOrder ? c + j + 1 : g.connSlot[j];
}

// Primary / equation indices of the fully compositional layout without wells
// (indices/include/indices/indices.hpp:30-45).
template <int NC>
struct Layout
{
    static constexpr int B = 3 * NC + 1;
    static constexpr int NPS = 3 * NC + 8;
    NZ_BOTH static int comp(int phase, int i) { return 1 + phase * (NC - 1) + i; }
    static constexpr int So = 3 * NC - 2;
    static constexpr int Sg = 3 * NC - 1;
    static constexpr int Sw = 3 * NC;
    // equations
    static constexpr int mass = 0;
    static constexpr int fugOG = NC;
    static constexpr int fugOW = 2 * NC;
    static constexpr int closure = 3 * NC;
    // phase-state record (PetscPhaseStateCodec)
    static constexpr int psFlag = 0;
    static constexpr int psKg = 1;
    static constexpr int psKw = 1 + NC;
    static constexpr int psZ = 1 + 2 * NC;
    static constexpr int psBeta = 1 + 3 * NC;
    static constexpr int psZf = 4 + 3 * NC;
    static constexpr int psSuppression = 7 + 3 * NC;
};

template <int NC, class S>
struct CellStateT
{
    S p, sat[3];
    S x[3][NC];
    uint8_t presence;
};

template <int NC, class S>
struct CellPropsT
{
    S density[3], viscosity[3], mobility[3], saturation[3];
    S w[3][NC];
    S f[3][NC];
    S porosity;
};

// Exterior values a face needs (frozen neighbour, face_flux.hpp:54-63).
template <int NC>
struct FaceSide
{
    double p;
    double density[3], saturation[3], mobility[3];
    double w[3][NC];
};

NZ_BOTH uint8_t decodePresence(double flag)
{
    const int raw = static_cast<int>(flag + (flag >= 0.0 ? 0.5 : -0.5));
    return (raw <= 0 || raw > 7) ? 0 : uint8_t(raw);
}

// CellStateCodec::decode with direction `k` seeded (k < 0: no direction).
template <int NC, class S>
NZ_HD void decodeCell(const double *primary, double flag, int k, CellStateT<NC, S> &st)
{
    using L = Layout<NC>;
    st.presence = decodePresence(flag);
    st.p = Seed<S>::at(primary[0], 0, k);
    for (int ph = 0; ph < 3; ++ph)
    {
        S dependent = S(1.0);
        for (int i = 0; i < NC - 1; ++i)
        {
            const int idx = L::comp(ph, i);
            st.x[ph][i] = Seed<S>::at(primary[idx], idx, k);
            dependent = dependent - st.x[ph][i];
        }
        const double dv = val(dependent);
        if (fabs(dv) <= kCancellationBoundary)
            dependent += -dv;
        st.x[ph][NC - 1] = dependent;
    }
    const int sIdx[3] = {L::So, L::Sg, L::Sw};
    for (int ph = 0; ph < 3; ++ph)
        st.sat[ph] = Seed<S>::at(primary[sIdx[ph]], sIdx[ph], k);
}

// ---- EOS in S (cubic_eos.hpp) -------------------------------------------
template <int NC, class S>
NZ_HD void mixingT(const FluidDev &F, const S &P, const S &T, bool aqueous, S (&A)[NC][NC], S (&Bi)[NC])
{
    S sqrtAi[NC];
    for (int i = 0; i < NC; ++i)
    {
        const S pr = P / F.pc[i];
        const S tr = T / F.tc[i];
        S alpha;
        if (F.eosModel == EOS_SW && i == F.water)
        {
            const S trw = T / F.tc[i];
            const double saltFactor = 1.0 - 0.0103 * ::pow(F.salinity, 1.1);
            const S sqrtAlpha = S(1.0) + 0.4530 * (S(1.0) - trw * saltFactor) + 0.0034 * (pow(trw, -3.0) - S(1.0));
            alpha = sqrtAlpha * sqrtAlpha;
        }
        else
        {
            const double omega = F.omega[i];
            double m = 0.37464 + 1.54226 * omega - 0.26992 * omega * omega;
            if (F.eosType == 5 && omega > 0.49)
                m = 0.379642 + 1.48503 * omega - 0.164423 * omega * omega + 0.016666 * omega * omega * omega;
            const S alphaRoot = S(1.0) + m * (S(1.0) - sqrt(tr));
            alpha = alphaRoot * alphaRoot;
        }
        const S reducedA = F.omegaA * alpha * pr / (tr * tr);
        sqrtAi[i] = sqrt(reducedA);
        Bi[i] = F.omegaB * pr / tr;
    }
    const bool swAq = F.eosModel == EOS_SW && aqueous;
    const double Tv = val(T);
    for (int i = 0; i < NC; ++i)
        for (int j = i; j < NC; ++j)
        {
            double kij = F.kij[i * kMaxNc + j];
            if (swAq)
                kij = swAqueousBip(F, i, j, Tv, F.salinity);
            const S aij = sqrtAi[i] * sqrtAi[j] * (1.0 - kij);
            A[i][j] = aij;
            A[j][i] = aij;
        }
}

template <int NC, class S>
NZ_HD void phaseMixT(const S (&x)[NC], const S (&A)[NC][NC], const S (&Bi)[NC], S (&Si)[NC], S &Am, S &Bm)
{
    Am = S(0.0);
    Bm = S(0.0);
    for (int i = 0; i < NC; ++i)
    {
        S si = S(0.0);
        for (int j = 0; j < NC; ++j)
            si += x[j] * A[i][j];
        Si[i] = si;
        Bm += x[i] * Bi[i];
    }
    for (int i = 0; i < NC; ++i)
        Am += x[i] * Si[i];
}

// solveCubic + liquidRoot / vaporRoot (cubic_eos.hpp:696-803); ok=false where the reference throws.
template <class S>
NZ_HD S cubicRootT(const S &A, const S &B, double m1, double m2, bool vapour, bool &ok)
{
    const S e0 = -(A * B + m1 * m2 * B * B * (B + 1.0));
    const S e1 = A - (m1 + m2 - m1 * m2) * B * B - (m1 + m2) * B;
    const S e2 = (m1 + m2 - 1.0) * B - 1.0;
    const S a = e2, b = e1, c = e0;
    const S Q = (a * a - 3.0 * b) / 9.0;
    const S R = (2.0 * a * a * a - 9.0 * a * b + 27.0 * c) / 54.0;
    const S disc = R * R - Q * Q * Q;
    S roots[3] = {S(nzNan()), S(nzNan()), S(nzNan())};
    if (val(disc) < 0.0)
    {
        S arg = R / sqrt(Q * Q * Q);
        if (val(arg) > 1.0)
            arg = S(1.0);
        else if (val(arg) < -1.0)
            arg = S(-1.0);
        const S theta = acos(arg);
        roots[0] = -2.0 * sqrt(Q) * cos(theta / 3.0) - a / 3.0;
        roots[1] = -2.0 * sqrt(Q) * cos((theta + 2.0 * kPi) / 3.0) - a / 3.0;
        roots[2] = -2.0 * sqrt(Q) * cos((theta - 2.0 * kPi) / 3.0) - a / 3.0;
    }
    else
    {
        S Sc;
        if (val(R) > 0.0)
            Sc = -pow(abs(R) + sqrt(disc), 1.0 / 3.0);
        else
            Sc = pow(abs(R) + sqrt(disc), 1.0 / 3.0);
        S Tt = S(0.0);
        if (fabs(val(Sc)) > 0.0)
            Tt = Q / Sc;
        roots[0] = Sc + Tt - a / 3.0;
    }
    for (int r = 0; r < 3; ++r)
        if (isfinite(val(roots[r])) && val(roots[r]) <= 0.0)
            roots[r] = S(nzNan());
    bool found = false;
    S best = S(nzNan());
    for (int r = 0; r < 3; ++r)
    {
        const double z = val(roots[r]);
        if (!isfinite(z) || !(z > val(B)))
            continue;
        if (!found || (vapour ? (z > val(best)) : (z < val(best))))
        {
            best = roots[r];
            found = true;
        }
    }
    ok = found;
    return best;
}

// fugacityAtRoot (cubic_eos.hpp:902-934): f_i = phi_i P x_i
template <int NC, class S>
NZ_HD bool fugacityT(const S &P, const S (&x)[NC], const S (&Bi)[NC], const S (&Si)[NC], const S &Am,
                     const S &Bm, const S &Z, double m1, double m2, S (&f)[NC])
{
    if (!(val(Bm) > 0.0) || !(val(Am) > 0.0) || !(val(Z - Bm) > 0.0))
        return false;
    const S commonA = -log(Z - Bm);
    const S logRatio = log((Z + m2 * Bm) / (Z + m1 * Bm));
    const S commonB = logRatio * Am / ((m1 - m2) * Bm);
    const S commonC = (Z - 1.0) / Bm;
    for (int i = 0; i < NC; ++i)
    {
        const S lnPhi = commonA + commonB * (2.0 * Si[i] / Am - Bi[i] / Bm) + Bi[i] * commonC;
        const S phi = exp(lnPhi);
        f[i] = phi * P * x[i];
    }
    return true;
}

// LBC viscosity at molar density rho (compositional_properties.hpp:106-150)
template <int NC, class S>
NZ_HD S lbcViscosityT(const FluidDev &F, const NatConst &K, const S (&x)[NC], const S &rho, const S &T)
{
    S num = S(0.0), den = S(0.0);
    for (int i = 0; i < NC; ++i)
    {
        const double mwSqrt = K.lbcMwSqrt[i];
        const S tr = T / F.tc[i];
        const double eps = K.lbcEps[i];
        const S cv = val(tr) > 1.5 ? 17.78e-5 * pow(4.58 * tr - 1.67, 0.625) / eps
                                   : 34.0e-5 * pow(tr, 0.94) / eps;
        num += x[i] * cv * mwSqrt;
        den += x[i] * mwSqrt;
    }
    const S atm = num / den;
    S pc = S(0.0), tc = S(0.0), vc = S(0.0), mw = S(0.0);
    for (int i = 0; i < NC; ++i)
    {
        pc += F.pc[i] * x[i];
        tc += F.tc[i] * x[i];
        vc += F.vc[i] * x[i];
        mw += F.mw[i] * x[i];
    }
    const S epsMix = 5.4402 * pow(tc / kKelvinPerRankine, 1.0 / 6.0) /
        (sqrt(1000.0 * mw) * pow(pc / kPsi, 2.0 / 3.0) * kCentipoise);
    const S r = vc * rho;
    const S r2 = r * r;
    const S r3 = r2 * r;
    const S r4 = r2 * r2;
    const S poly = 0.1023 + 0.023364 * r + 0.058533 * r2 + (-0.040758) * r3 + 0.0093324 * r4;
    const S poly2 = poly * poly;
    const S poly4 = poly2 * poly2;
    return atm + (poly4 + (-1.0e-4)) / epsMix;
}

// benchmark_common.hpp:97-126 quadratic curves
template <class S>
NZ_HD S krWater(const NatConst &K, const S &sw)
{
    const double v = val(sw);
    if (v <= K.swc) return S(0.0);
    if (v >= 1.0 - K.sorw) return S(K.krwMax);
    const S se = (sw - K.swc) / (1.0 - K.swc - K.sorw);
    return S(K.krwMax) * se * se;
}
template <class S>
NZ_HD S krGas(const NatConst &K, const S &sg)
{
    const double v = val(sg);
    if (v <= K.sgc) return S(0.0);
    if (v >= 1.0 - K.sorg - K.swc) return S(K.krgMax);
    const S se = (sg - K.sgc) / (1.0 - K.sorg - K.swc - K.sgc);
    return S(K.krgMax) * se * se;
}
template <class S>
NZ_HD S krOil(const NatConst &K, const S &so)
{
    const double v = val(so);
    if (v <= K.sorg) return S(0.0);
    if (v >= 1.0 - K.swc) return S(K.kroMax);
    const S se = (so - K.sorg) / (1.0 - K.swc - K.sorg);
    return S(K.kroMax) * se * se;
}

// evaluateFullyCompositional_ for PR / SW (cell_property_evaluator.hpp:236-393).
template <int NC, class S>
NZ_HD bool cellProperties(const FluidDev &F, const NatConst &K, const CellStateT<NC, S> &st, double porosity,
                          CellPropsT<NC, S> &pr)
{
    pr.porosity = S(porosity);
    S comp[3][NC];
    for (int ph = 0; ph < 3; ++ph)
        for (int i = 0; i < NC; ++i)
            comp[ph][i] = st.x[ph][i];
    if (!(st.presence & WATER_BIT))
    {
        // absent water phase evaluated at pure H2O (:263-281)
        for (int i = 0; i < NC; ++i)
            comp[2][i] = S(0.0);
        comp[2][F.water] = S(1.0);
    }
    const S T = S(K.temperature);
    S A[NC][NC], Bi[NC];
    if (F.eosModel != EOS_CPA)
        mixingT<NC, S>(F, st.p, T, false, A, Bi);
    for (int ph = 0; ph < 3; ++ph)
    {
        pr.saturation[ph] = st.sat[ph];
        S Aw[NC][NC], Bw[NC];
        const bool aq = ph == WATER && F.eosModel == EOS_SW;
        if (aq)
            mixingT<NC, S>(F, st.p, T, true, Aw, Bw);
        const S(&Ap)[NC][NC] = aq ? Aw : A;
        const S(&Bp)[NC] = aq ? Bw : Bi;
        S Z;
        if (F.eosModel == EOS_CPA)
        {
            // CPA keeps the full phaseResult path per phase (:336-352)
            S phi[NC];
            if (cpaPhaseT<NC, S>(F, st.p, K.temperature, comp[ph], ph != GAS, Z, phi) != ERR_NONE)
                return false;
            for (int i = 0; i < NC; ++i)
                pr.f[ph][i] = phi[i] * st.p * comp[ph][i];
        }
        else
        {
            S Si[NC], Am, Bm;
            phaseMixT<NC, S>(comp[ph], Ap, Bp, Si, Am, Bm);
            bool ok = true;
            Z = cubicRootT<S>(Am, Bm, F.m1, F.m2, ph == GAS, ok);
            if (!ok || !fugacityT<NC, S>(st.p, comp[ph], Bp, Si, Am, Bm, Z, F.m1, F.m2, pr.f[ph]))
                return false;
        }
        // eosFlowProperties (fluid_system.hpp:99-125), no volume translation
        S total = S(0.0);
        for (int i = 0; i < NC; ++i)
        {
            pr.w[ph][i] = comp[ph][i] * F.mw[i];
            total += pr.w[ph][i];
        }
        if (!(val(total) > 0.0))
            return false;
        for (int i = 0; i < NC; ++i)
            pr.w[ph][i] = pr.w[ph][i] / total;
        const S rhoMolar = st.p / (kGasConstant * T * Z);
        S mwMix = S(0.0);
        for (int i = 0; i < NC; ++i)
            mwMix += comp[ph][i] * F.mw[i];
        pr.density[ph] = rhoMolar * mwMix;
        pr.viscosity[ph] = lbcViscosityT<NC, S>(F, K, comp[ph], rhoMolar, T);
    }
    S sgRelperm = st.sat[GAS];
    if (!(st.presence & GAS_BIT))
        clearDer(sgRelperm);
    const S freeGas = sgRelperm - S(0.0);
    const S kr[3] = {krOil<S>(K, st.sat[OIL]), krGas<S>(K, freeGas), krWater<S>(K, st.sat[WATER])};
    for (int ph = 0; ph < 3; ++ph)
        pr.mobility[ph] = (st.presence & bitOf(ph)) ? kr[ph] / pr.viscosity[ph] : S(0.0);
    return true;
}

// computeFluidComponentAccumulation (accumulation.hpp:30-78)
template <int NC, class S>
NZ_HD S accumulation(const CellPropsT<NC, S> &pr, int c)
{
    S mass = S(0.0);
    for (int ph = 0; ph < 3; ++ph)
        mass += pr.density[ph] * pr.saturation[ph] * pr.w[ph][c];
    return pr.porosity * mass;
}

// assembleCellLocalResidual (cell_residual.hpp:73-320), fully compositional branch.
template <int NC, class S>
NZ_HD void localResidual(const NatConst &K, const CellStateT<NC, S> &st, const CellPropsT<NC, S> &pr,
                         const double *prevAccumulation, double volume, S (&res)[3 * NC + 1])
{
    using L = Layout<NC>;
    const double storage = volume / K.timeStep;
    for (int c = 0; c < NC; ++c)
        res[L::mass + c] = (accumulation<NC, S>(pr, c) - prevAccumulation[c]) * storage;
    const bool oil = st.presence & OIL_BIT, gas = st.presence & GAS_BIT, water = st.presence & WATER_BIT;
    auto fugBlock = [&](int eqBegin, int ref, int other, int altRef, bool altActive) {
        for (int c = 0; c < NC; ++c)
        {
            const int eq = eqBegin + c;
            const bool refTrace = val(st.x[ref][c]) <= kTraceComposition;
            const bool otherTrace = val(st.x[other][c]) <= kTraceComposition;
            if (otherTrace)
            {
                res[eq] = st.x[other][c];
                continue;
            }
            if (refTrace)
            {
                if (altActive && altRef >= 0 && val(st.x[altRef][c]) > kTraceComposition)
                {
                    res[eq] = (pr.f[altRef][c] - pr.f[other][c]) / kBar / K.fugacityScaling;
                    continue;
                }
                res[eq] = st.x[ref][c];
                continue;
            }
            res[eq] = (pr.f[ref][c] - pr.f[other][c]) / kBar / K.fugacityScaling;
        }
    };
    auto inactiveBlock = [&](int eqBegin, int phase) {
        for (int c = 0; c < NC - 1; ++c)
            res[eqBegin + c] = st.x[phase][c] - val(st.x[phase][c]);
        res[eqBegin + NC - 1] = st.sat[phase];
    };
    if (oil)
    {
        if (gas)
            fugBlock(L::fugOG, OIL, GAS, -1, false);
        else
            inactiveBlock(L::fugOG, GAS);
        if (water)
            fugBlock(L::fugOW, OIL, WATER, GAS, gas);
        else
            inactiveBlock(L::fugOW, WATER);
    }
    else
    {
        inactiveBlock(L::fugOG, OIL);
        if (gas && water)
            fugBlock(L::fugOW, GAS, WATER, -1, false);
        else if (gas)
            inactiveBlock(L::fugOW, WATER);
        else
            inactiveBlock(L::fugOW, GAS);
    }
    res[L::closure] = st.sat[OIL] + st.sat[GAS] + st.sat[WATER] - 1.0;
}

// chooseUpwindSide (face_flux.hpp:65-87): true = interior upwind
NZ_HDI bool interiorUpwind(double dPhi, double volIn, double volEx, long long idIn, long long idEx)
{
    if (dPhi > 0.0) return false;
    if (dPhi < 0.0) return true;
    if (volIn > volEx) return true;
    if (volEx > volIn) return false;
    return idIn < idEx;
}

// computeFaceMassFlux with the exterior frozen (face_flux.hpp:174-321):
// outward mass rate of every component from the interior cell.
template <int NC, class S>
NZ_HD void faceFlux(const CellStateT<NC, S> &st, const CellPropsT<NC, S> &in, const FaceSide<NC> &ex,
                    double trans, double gdz, double volIn, double volEx, long long idIn, long long idEx,
                    S (&out)[NC])
{
    for (int c = 0; c < NC; ++c)
        out[c] = S(0.0);
    for (int ph = 0; ph < 3; ++ph)
    {
        const S &rhoIn = in.density[ph];
        const S &satIn = in.saturation[ph];
        const S satAvg = 0.5 * (satIn + ex.saturation[ph]);
        const S avgDensity = 0.5 * (rhoIn * satIn + ex.density[ph] * ex.saturation[ph]) / smax(val(satAvg), 1.0e-8);
        const S dPhi = ex.p + avgDensity * gdz - st.p;
        const bool inUp = interiorUpwind(val(dPhi), volIn, volEx, idIn, idEx);
        S rate;
        if (inUp)
        {
            const S darcy = -trans * dPhi * in.mobility[ph];
            rate = darcy * in.density[ph];
        }
        else
        {
            const S darcy = -trans * dPhi * ex.mobility[ph];
            rate = darcy * ex.density[ph];
        }
        for (int c = 0; c < NC; ++c)
            out[c] += inUp ? rate * in.w[ph][c] : rate * ex.w[ph][c];
    }
}

// computeFaceMassFluxValue (face_flux.hpp:330-430): the residual's pure-FP64
// face kernel on both sides' values.
template <int NC>
NZ_HD void faceFluxValue(const FaceSide<NC> &in, const FaceSide<NC> &ex, double trans, double gdz, double volIn,
                         double volEx, long long idIn, long long idEx, double (&out)[NC])
{
    for (int c = 0; c < NC; ++c)
        out[c] = 0.0;
    for (int ph = 0; ph < 3; ++ph)
    {
        const double rhoIn = in.density[ph], rhoEx = ex.density[ph];
        const double satIn = in.saturation[ph], satEx = ex.saturation[ph];
        const double avgDensity = 0.5 * (rhoIn * satIn + rhoEx * satEx) / smax(0.5 * (satIn + satEx), 1.0e-8);
        const double dPhi = ex.p + avgDensity * gdz - in.p;
        const bool inUp = interiorUpwind(dPhi, volIn, volEx, idIn, idEx);
        const double mobility = inUp ? in.mobility[ph] : ex.mobility[ph];
        const double density = inUp ? in.density[ph] : ex.density[ph];
        const double rate = -trans * dPhi * mobility * density;
        for (int c = 0; c < NC; ++c)
            out[c] += rate * (inUp ? in.w[ph][c] : ex.w[ph][c]);
    }
}

} // namespace nz
