// natural_state.cuh -- the Natural phase-state transaction of one cell.
//
// Restates FullyCompositionalThreePhaseEquilibrium
// (models/include/natural/state/three_phase_equilibrium.hpp):
//   sanitizePrimaryBeforeFlash      :505-553
//   updatePhaseState                :282-503
//   updateSecondary                 :164-280
//   assignFlashResult               :128-162
//   assignCanonicalSingleNonaqueousReducedSet_ :642-696
//   hasStrongMissingPhaseInstability_           :698-722
//   canonicalizeSwNonAqueousRoles_  :566-627
// on top of the device flash solver.  A thrown exception of the reference
// becomes a recoverable failure of the cell (the runtime rolls every cell
// back, natural_petsc_runtime_state.inc:243-300).
#pragma once

#include "flash.cuh"
#include "natural.cuh"

namespace nz
{

template <int NC>
struct PhaseRec
{
    uint8_t presence;
    uint8_t suppression;
    double Kg[NC], Kw[NC], z[NC], beta[3], Z[3];
};

constexpr int UPD_UPDATED = 0;
constexpr int UPD_STABLE_REDUCED = 1;
constexpr int UPD_FAILED = 2;

struct UpdateOutcome
{
    int status;
    bool phaseRemoved, missingPhaseUnstable, stabilityInvalid, restrictedFailed, unrestrictedFailed;
};

template <int NC>
NZ_HD bool decodePhaseRec(const double *ps, PhaseRec<NC> &r)
{
    using L = Layout<NC>;
    r.presence = decodePresence(ps[L::psFlag]);
    r.suppression = uint8_t(static_cast<int>(ps[L::psSuppression] + 0.5)) & ALL_BITS;
    for (int i = 0; i < NC; ++i)
    {
        r.Kg[i] = ps[L::psKg + i];
        r.Kw[i] = ps[L::psKw + i];
        r.z[i] = ps[L::psZ + i];
    }
    for (int p = 0; p < 3; ++p)
    {
        r.beta[p] = ps[L::psBeta + p];
        r.Z[p] = ps[L::psZf + p];
    }
    return r.presence != 0;
}

template <int NC>
NZ_HD void encodePhaseRec(const PhaseRec<NC> &r, double *ps)
{
    using L = Layout<NC>;
    ps[L::psFlag] = double(r.presence);
    for (int i = 0; i < NC; ++i)
    {
        ps[L::psKg + i] = r.Kg[i];
        ps[L::psKw + i] = r.Kw[i];
        ps[L::psZ + i] = r.z[i];
    }
    for (int p = 0; p < 3; ++p)
    {
        ps[L::psBeta + p] = r.beta[p];
        ps[L::psZf + p] = r.Z[p];
    }
    ps[L::psSuppression] = double(r.suppression);
}

// Result of the part of updatePhaseState before its first flash or test.
template <int NC>
struct UpdateHead
{
    double P;
    double zt[NC];
    double comps[3][NC];
    uint8_t active;
    uint8_t suppression;   // the phase state's suppression flags after the head
    bool removed;
};

template <int NC>
struct Equilibrium
{
    Solver<NC> s;
    const NatConst *K;
    using L = Layout<NC>;

    NZ_HD double floor() const { return s.O().floor; }
    NZ_HD static int satIndex(int phase) { return phase == OIL ? L::So : (phase == GAS ? L::Sg : L::Sw); }

    // three_phase_detail::normalize (:23-35)
    NZ_HD void normalizeFloor(double *x)
    {
        double sum = 0.0;
        for (int i = 0; i < NC; ++i)
        {
            x[i] = smax(x[i], floor());
            sum += x[i];
        }
        if (!(sum > 0.0) || !isfinite(sum))
            s.fail(ERR_EOS);
        for (int i = 0; i < NC; ++i)
            x[i] /= sum;
    }

    NZ_HD void phaseCompositions(const double *primary, double (&c)[3][NC])
    {
        for (int ph = 0; ph < 3; ++ph)
        {
            c[ph][NC - 1] = 1.0;
            for (int i = 0; i < NC - 1; ++i)
            {
                c[ph][i] = primary[L::comp(ph, i)];
                c[ph][NC - 1] -= c[ph][i];
            }
            normalizeFloor(c[ph]);
        }
    }

    NZ_HD void writeComposition(double *primary, const double *x, int phase)
    {
        for (int i = 0; i < NC - 1; ++i)
            primary[L::comp(phase, i)] = x[i];
    }

    // sanitizePrimaryBeforeFlash without variable bounds (:505-553)
    NZ_HD void sanitize(double *primary)
    {
        for (int ph = 0; ph < 3; ++ph)
        {
            double sum = 0.0;
            for (int i = 0; i < NC - 1; ++i)
            {
                double &v = primary[L::comp(ph, i)];
                v = sclamp(v, floor(), 1.0 - floor());
                sum += v;
            }
            const double maxSum = 1.0 - floor();
            if (sum > maxSum)
            {
                const double scale = maxSum / sum;
                for (int i = 0; i < NC - 1; ++i)
                    primary[L::comp(ph, i)] *= scale;
            }
        }
    }

    // transitionOverallComposition_ (:763-788)
    NZ_HD void transitionOverall(const double *primary, const PhaseRec<NC> &ps, double *z)
    {
        double c[3][NC];
        phaseCompositions(primary, c);
        for (int i = 0; i < NC; ++i)
            z[i] = 0.0;
        double betaSum = 0.0;
        for (int ph = 0; ph < 3; ++ph)
        {
            if (!(ps.presence & bitOf(ph)))
                continue;
            const double beta = smax(ps.beta[ph], 0.0);
            betaSum += beta;
            for (int i = 0; i < NC; ++i)
                z[i] += beta * c[ph][i];
        }
        if (!(betaSum > 1.0e-14))
        {
            for (int i = 0; i < NC; ++i)
                z[i] = ps.z[i];
            return;
        }
        for (int i = 0; i < NC; ++i)
            z[i] /= betaSum;
        normalizeFloor(z);
    }

    // assignFlashResult (:128-162)
    NZ_HD void assignFlashResult(double *primary, PhaseRec<NC> &ps, const Result<NC> &f)
    {
        if (!f.converged)
        {
            s.fail(ERR_EOS);
            return;
        }
        primary[L::So] = f.sat[0];
        primary[L::Sg] = f.sat[1];
        primary[L::Sw] = f.sat[2];
        for (int ph = 0; ph < 3; ++ph)
            writeComposition(primary, f.x[ph], ph);
        ps.presence = f.presence;
        for (int ph = 0; ph < 3; ++ph)
            if (f.presence & bitOf(ph))
                ps.suppression &= uint8_t(~bitOf(ph));
        double z[NC];
        for (int i = 0; i < NC; ++i)
            z[i] = 0.0;
        for (int ph = 0; ph < 3; ++ph)
            for (int i = 0; i < NC; ++i)
                z[i] += f.beta[ph] * f.x[ph][i];
        normalizeFloor(z);
        for (int i = 0; i < NC; ++i)
        {
            ps.z[i] = z[i];
            ps.Kg[i] = f.Kg[i];
            ps.Kw[i] = f.Kw[i];
        }
        for (int ph = 0; ph < 3; ++ph)
        {
            ps.beta[ph] = f.beta[ph];
            ps.Z[ph] = f.Z[ph];
        }
    }

    // updateSecondary (:164-280)
    NZ_HD void updateSecondary(double *primary, PhaseRec<NC> &ps)
    {
        double c[3][NC];
        phaseCompositions(primary, c);
        const double sat[3] = {primary[L::So], primary[L::Sg], primary[L::Sw]};
        const double p = primary[0];
        const double T = K->temperature;
        double amount[3] = {0.0, 0.0, 0.0};
        double total = 0.0;
        s.ensureCache(p, T);
        for (int ph = 0; ph < 3; ++ph)
        {
            if (!(ps.presence & bitOf(ph)))
                continue;
            double z;
            if (s.F->eosModel == EOS_CPA)
            {
                // eos.compressibility's CPA branch: Z = p / (rho R T) at the
                // density root (cubic_eos.hpp:865-884)
                CpaMix<NC> cm;
                cpaMixing<NC>(*s.F, T, c[ph], cm);
                double rho = 0.0;
                const int rc = cpaDensityRoot<NC>(*s.F, p, T, c[ph], ph != GAS, cm, rho);
                if (rc != ERR_NONE)
                {
                    s.fail(rc);
                    return;
                }
                z = p / (rho * kGasConstant * T);
            }
            else
            {
                const MixParams<NC> &mp = (ph == WATER && s.sw()) ? s.aq : s.nonAq;
                PhaseMix<NC> m;
                phaseMixing<NC>(c[ph], mp, m);
                z = selectCubicRoot(m.A, m.B, s.F->m1, s.F->m2, ph == GAS);
            }
            if (!isfinite(z))
            {
                s.fail(ERR_EOS);
                return;
            }
            ps.Z[ph] = z;
            const double rho = molarDensity(p, T, z);
            amount[ph] = rho * smax(sat[ph], 0.0);
            total += amount[ph];
        }
        if (!(total > 1.0e-14))
        {
            s.fail(ERR_EOS);
            return;
        }
        for (int i = 0; i < NC; ++i)
            ps.z[i] = 0.0;
        for (int ph = 0; ph < 3; ++ph)
        {
            ps.beta[ph] = amount[ph] / total;
            for (int i = 0; i < NC; ++i)
                ps.z[i] += ps.beta[ph] * c[ph][i];
        }
        normalizeFloor(ps.z);
        if ((ps.presence & OIL_BIT) && (ps.presence & GAS_BIT))
            for (int i = 0; i < NC; ++i)
                ps.Kg[i] = c[1][i] / smax(c[0][i], floor());
        if ((ps.presence & OIL_BIT) && (ps.presence & WATER_BIT))
            for (int i = 0; i < NC; ++i)
                ps.Kw[i] = c[2][i] / smax(c[0][i], floor());
    }

    // Wilson-volatility role of one nonaqueous composition (:629-640)
    NZ_HD int expectedRole(double pressure, const double *x) const
    {
        double volatility = 0.0, magnitude = 0.0;
        for (int i = 0; i < NC; ++i)
        {
            const double lnK = log(s.F->pc[i] / pressure) +
                5.373 * (1.0 + s.F->omega[i]) * (1.0 - s.F->tc[i] / K->temperature);
            const double term = x[i] * lnK;
            volatility += term;
            magnitude += fabs(term);
        }
        return volatility >= -1.0e-10 * smax(1.0, magnitude) ? GAS : OIL;
    }

    // assignCanonicalSingleNonaqueousReducedSet_ (:642-696)
    NZ_HD bool canonicalSingleNonaqueous(double *primary, PhaseRec<NC> &ps, const double *z, uint8_t active,
                                         double (&seed)[3][NC])
    {
        if (s.sw())
            return false;
        const bool hasOil = active & OIL_BIT, hasGas = active & GAS_BIT;
        if (hasOil == hasGas)
            return false;
        const int act = hasOil ? OIL : GAS;
        const int expected = expectedRole(primary[0], seed[act]);
        if (expected == act)
            return false;
        uint8_t corrected = uint8_t((active & ~bitOf(act)) | bitOf(expected));
        for (int i = 0; i < NC; ++i)
            seed[expected][i] = seed[act][i];
        Result<NC> canonical;
        s.flashRestricted(primary[0], K->temperature, z, corrected, &seed, canonical);
        if (!canonical.converged || canonical.presence != corrected || s.err)
            return false;
        assignFlashResult(primary, ps, canonical);
        return !s.err;
    }

    NZ_HD static bool strongInstability(const StabilityResult<NC> &st, uint8_t present, uint8_t suppression)
    {
        if (!st.valid)
            return false;
        for (int ph = 0; ph < 3; ++ph)
        {
            if (present & bitOf(ph))
                continue;
            const double margin = (suppression & bitOf(ph)) ? 1.0e-4 : 1.0e-6;
            if (st.unstable[ph] && st.trialSum[ph] > 1.0 + margin)
                return true;
        }
        return false;
    }

    // canonicalizeSwNonAqueousRoles_ (:566-627)
    NZ_HD void canonicalizeSwRoles(double *primary, PhaseRec<NC> &ps)
    {
        if (!s.sw() || !(ps.presence & OIL_BIT) || !(ps.presence & GAS_BIT))
            return;
        double c[3][NC];
        phaseCompositions(primary, c);
        const double pressure = primary[0];
        double orientation = 0.0, magnitude = 0.0;
        for (int i = 0; i < NC; ++i)
        {
            const double lnK = log(s.F->pc[i] / pressure) +
                5.373 * (1.0 + s.F->omega[i]) * (1.0 - s.F->tc[i] / K->temperature);
            const double term = (c[1][i] - c[0][i]) * lnK;
            orientation += term;
            magnitude += fabs(term);
        }
        if (orientation >= -1.0e-10 * smax(1.0, magnitude))
            return;
        double t = primary[L::So];
        primary[L::So] = primary[L::Sg];
        primary[L::Sg] = t;
        for (int i = 0; i < NC - 1; ++i)
        {
            t = primary[L::comp(OIL, i)];
            primary[L::comp(OIL, i)] = primary[L::comp(GAS, i)];
            primary[L::comp(GAS, i)] = t;
        }
        t = ps.beta[0];
        ps.beta[0] = ps.beta[1];
        ps.beta[1] = t;
        t = ps.Z[0];
        ps.Z[0] = ps.Z[1];
        ps.Z[1] = t;
        double cc[3][NC];
        phaseCompositions(primary, cc);
        for (int i = 0; i < NC; ++i)
        {
            ps.Kg[i] = cc[1][i] / smax(cc[0][i], floor());
            if (ps.presence & WATER_BIT)
                ps.Kw[i] = cc[2][i] / smax(cc[0][i], floor());
        }
    }

    // The part of updatePhaseState (:282-335) before any flash or stability
    // test: SW role orientation, the overall composition, removal of phases
    // whose Newton saturation fell to 1e-4 and the present phases'
    // compositions.  False when a composition cannot be normalised.
    NZ_HDN bool updateHead(double *primary, PhaseRec<NC> &ps, UpdateHead<NC> &h)
    {
        canonicalizeSwRoles(primary, ps);
        transitionOverall(primary, ps, h.zt);
        uint8_t active = ps.presence;
        ps.suppression &= uint8_t(~active);
        bool removed = false;
        const double newtonSat[3] = {primary[L::So], primary[L::Sg], primary[L::Sw]};
        for (int ph = 0; ph < 3; ++ph)
            if ((active & bitOf(ph)) && newtonSat[ph] <= 1.0e-4)
            {
                active &= uint8_t(~bitOf(ph));
                ps.suppression |= uint8_t(bitOf(ph));
                primary[satIndex(ph)] = 0.0;
                removed = true;
            }
        if (active == 0)
        {
            int survivor = 0;
            for (int ph = 1; ph < 3; ++ph)
                if (newtonSat[survivor] < newtonSat[ph])
                    survivor = ph;
            active |= uint8_t(bitOf(survivor));
            ps.suppression &= uint8_t(~bitOf(survivor));
            primary[satIndex(survivor)] = 1.0;
            removed = true;
        }
        h.active = active;
        h.removed = removed;
        ps.presence = active;
        for (int i = 0; i < NC; ++i)
            ps.z[i] = h.zt[i];
        phaseCompositions(primary, h.comps);
        h.P = primary[0];
        h.suppression = ps.suppression;
        return !s.err;
    }

    // updatePhaseState (:282-503).  On failure the caller keeps its originals.
    NZ_HDN UpdateOutcome update(double *primary, PhaseRec<NC> &ps)
    {
        UpdateOutcome out{UPD_UPDATED, false, false, false, false, false};
        const double T = K->temperature;
        UpdateHead<NC> h;
        const bool headOk = updateHead(primary, ps, h);
        out.phaseRemoved = h.removed;
        if (!headOk)
        {
            out.status = UPD_FAILED;
            return out;
        }
        const double *zt = h.zt;
        uint8_t active = h.active;
        const bool removed = h.removed;
        double (&comps)[3][NC] = h.comps;
        const double P = primary[0];
        if (removed)
        {
            Result<NC> reduced;
            s.flashRestricted(P, T, zt, active, &comps, reduced);
            if (reduced.converged && !s.err)
            {
                bool unstableMissing = false;
                if (popcount3(reduced.presence) < 3)
                {
                    StabilityResult<NC> st;
                    s.stabilityTest(P, T, zt, reduced.presence, reduced.x, st);
                    if (!st.valid)
                    {
                        out.stabilityInvalid = true;
                        unstableMissing = true;
                    }
                    else
                    {
                        unstableMissing = strongInstability(st, reduced.presence, ps.suppression);
                        out.missingPhaseUnstable = unstableMissing;
                    }
                }
                if (!unstableMissing && !s.err)
                {
                    if (canonicalSingleNonaqueous(primary, ps, zt, reduced.presence, reduced.x))
                    {
                        out.status = UPD_STABLE_REDUCED;
                        out.phaseRemoved = true;
                        return out;
                    }
                    if (s.err)
                    {
                        out.status = UPD_FAILED;
                        return out;
                    }
                    assignFlashResult(primary, ps, reduced);
                    out.status = s.err ? UPD_FAILED : UPD_STABLE_REDUCED;
                    out.phaseRemoved = true;
                    return out;
                }
            }
            if (s.err)
            {
                out.status = UPD_FAILED;
                return out;
            }
            Result<NC> reflashed;
            s.template flash<true>(P, T, zt, reflashed);
            if (reflashed.converged && !s.err)
            {
                assignFlashResult(primary, ps, reflashed);
                out.phaseRemoved = true;
                out.status = s.err ? UPD_FAILED : UPD_UPDATED;
                return out;
            }
            out.phaseRemoved = true;
            out.restrictedFailed = !reduced.converged;
            out.unrestrictedFailed = true;
            out.status = UPD_FAILED;
            return out;
        }
        else if (popcount3(active) < 3)
        {
            StabilityResult<NC> st;
            s.stabilityTest(P, T, zt, active, comps, st);
            if (s.err)
            {
                out.status = UPD_FAILED;
                return out;
            }
            const bool invalid = !st.valid;
            const bool unstable = !invalid && strongInstability(st, active, ps.suppression);
            if (invalid || unstable)
            {
                out.stabilityInvalid = invalid;
                out.missingPhaseUnstable = unstable;
                Result<NC> reflashed;
                s.template flash<true>(P, T, zt, reflashed);
                if (reflashed.converged && !s.err)
                {
                    assignFlashResult(primary, ps, reflashed);
                    out.status = s.err ? UPD_FAILED : UPD_UPDATED;
                    return out;
                }
                out.unrestrictedFailed = true;
                out.status = UPD_FAILED;
                return out;
            }
        }
        if (popcount3(active) < 3 && canonicalSingleNonaqueous(primary, ps, zt, active, comps))
        {
            out.status = UPD_STABLE_REDUCED;
            return out;
        }
        if (s.err)
        {
            out.status = UPD_FAILED;
            return out;
        }
        for (int ph = 0; ph < 3; ++ph)
        {
            if (ps.presence & bitOf(ph))
                continue;
            primary[satIndex(ph)] = 0.0;
            writeComposition(primary, zt, ph);
        }
        updateSecondary(primary, ps);
        if (s.err)
        {
            out.status = UPD_FAILED;
            return out;
        }
        if (popcount3(ps.presence) < 3)
            out.status = UPD_STABLE_REDUCED;
        return out;
    }
};

} // namespace nz
