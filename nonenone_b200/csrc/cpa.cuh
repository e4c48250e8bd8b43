// cpa.cuh -- cubic-plus-association phase evaluation (FP64), device and host.
//
// Restates CubicEquationOfState's CPA backend (models/include/natural/thermo/cubic_eos.hpp):
//   cpaMixing_                 :1417-1539  (temperature parameters + composition mixing)
//   cpaRadialDistribution_     :1541-1559
//   cpaAssociationDelta_       :1561-1582
//   cpaAssociationState_       :1584-2048  (the analytic single-symmetric-component path
//                                           and the single-donor safeguarded Newton; the
//                                           general multi-donor path reports ERR_NOT_PORTED)
//   cpaPressureAtDensityWithMix_ :2050-2078
//   cpaDensityRootValueWithMix_  :2090-2178 (bracket + bisection)
//   cpaDensityRoot_              :2191-2248 (two implicit corrections)
//   cpaAtDensity_                :2250-2307 (Z and ln phi)
//   cpaPhaseResult_              :2309-2370 (without the Gibbs-minimum root choice, which
//                                           the flash does not ask for)
// Every arithmetic expression keeps the reference's order of operations.
// Functions return ERR_NONE, or the error the reference would throw
// (ERR_EOS for std::runtime_error).
#pragma once

#include "eos.cuh"

namespace nz
{

constexpr double kSqrtTwo = 1.4142135623730950488;

template <int NC>
struct CpaMix
{
    double ai[NC], bi[NC], Si[NC];
    double aij[NC][NC];
    double factor[NC][NC];   // exp(epsilon / RT) - 1 of each donor/acceptor pair
    double volume[NC][NC];   // association volume of each donor/acceptor pair
    double a, b;
};

template <int NC>
struct CpaAssoc
{
    double donorX[NC], acceptorX[NC];
    double g, gPrimeOverG, bonded;
};

template <int NC>
NZ_HD void cpaMixing(const FluidDev &F, double T, const double *x, CpaMix<NC> &m)
{
    const CpaDev &o = F.cpa;
    double sqrtAi[NC];
    for (int i = 0; i < NC; ++i)
    {
        const double tr = T / F.tc[i];
        const double alphaRoot = 1.0 + o.c1[i] * (1.0 - sqrt(tr));
        m.ai[i] = o.a0[i] * alphaRoot * alphaRoot;
        m.bi[i] = o.b[i];
        sqrtAi[i] = sqrt(m.ai[i]);
    }
    for (int i = 0; i < NC; ++i)
        for (int j = 0; j < NC; ++j)
        {
            m.aij[i][j] = sqrtAi[i] * sqrtAi[j] * (1.0 - F.kij[i * kMaxNc + j]);
            m.factor[i][j] = 0.0;
            m.volume[i][j] = 0.0;
            if (o.donor[i] <= 0 || o.acceptor[j] <= 0)
                continue;
            double epsilon = o.crossEpsilon[i * kMaxNc + j];
            double beta = o.crossBeta[i * kMaxNc + j];
            if (!(epsilon > 0.0) || !(beta > 0.0))
            {
                if (o.epsilon[i] > 0.0 && o.epsilon[j] > 0.0 && o.beta[i] > 0.0 && o.beta[j] > 0.0)
                {
                    epsilon = 0.5 * (o.epsilon[i] + o.epsilon[j]);
                    beta = sqrt(o.beta[i] * o.beta[j]);
                }
                else
                {
                    epsilon = 0.0;
                    beta = 0.0;
                }
            }
            if (epsilon > 0.0 && beta > 0.0)
            {
                m.factor[i][j] = exp(epsilon / (kGasConstant * T)) - 1.0;
                m.volume[i][j] = beta;
            }
        }
    m.a = 0.0;
    m.b = 0.0;
    for (int i = 0; i < NC; ++i)
    {
        m.Si[i] = 0.0;
        for (int j = 0; j < NC; ++j)
            m.Si[i] += x[j] * m.aij[i][j];
        m.a += x[i] * m.Si[i];
        m.b += x[i] * m.bi[i];
    }
}

NZ_HDI void cpaRadial(const FluidDev &F, double eta, double &g, double &gPrimeOverG)
{
    if (!F.cpa.carnahanStarling)
    {
        const double denominator = 1.0 - 1.9 * eta;
        g = 1.0 / denominator;
        gPrimeOverG = 1.9 * g;
        return;
    }
    const double oneMinusEta = 1.0 - eta;
    g = (1.0 - 0.5 * eta) / (oneMinusEta * oneMinusEta * oneMinusEta);
    const double gPrime = (2.5 - eta) / (oneMinusEta * oneMinusEta * oneMinusEta * oneMinusEta);
    gPrimeOverG = gPrime / g;
}

template <int NC>
NZ_HDI double cpaDelta(int donor, int acceptor, const CpaMix<NC> &m, double g)
{
    const double temperatureFactor = m.factor[donor][acceptor];
    const double beta = m.volume[donor][acceptor];
    if (!(temperatureFactor > 0.0) || !(beta > 0.0))
        return 0.0;
    const double bij = 0.5 * (m.bi[donor] + m.bi[acceptor]);
    return g * temperatureFactor * bij * beta;
}

// cpaAssociationState_ (cubic_eos.hpp:1584-2048).
template <int NC>
NZ_HD int cpaAssociation(const FluidDev &F, double rho, const double *x, const CpaMix<NC> &m, CpaAssoc<NC> &s)
{
    const CpaDev &o = F.cpa;
    for (int i = 0; i < NC; ++i)
    {
        s.donorX[i] = 1.0;
        s.acceptorX[i] = 1.0;
    }
    const double eta = m.b * rho / 4.0;
    cpaRadial(F, eta, s.g, s.gPrimeOverG);
    if (o.symmetric >= 0)
    {
        // one associating component with equal donor and acceptor sites:
        // A X^2 + X - 1 = 0 with A = rho x n Delta
        const int k = o.symmetric;
        const int sites = o.donor[k];
        const double delta = cpaDelta<NC>(k, k, m, s.g);
        const double A = rho * x[k] * static_cast<double>(sites) * delta;
        const double X = 2.0 / (1.0 + sqrt(1.0 + 4.0 * A));
        s.donorX[k] = X;
        s.acceptorX[k] = X;
    }
    else if (o.singleDonor >= 0)
    {
        // one donor-bearing component: X_D (1 + sum_j A_j / (1 + B_j X_D)) = 1,
        // safeguarded Newton inside the bracket [0, 1]
        const int d = o.singleDonor;
        double aC[NC], bC[NC];
        double aSum = 0.0;
        for (int j = 0; j < NC; ++j)
        {
            aC[j] = 0.0;
            bC[j] = 0.0;
            if (o.acceptor[j] <= 0)
                continue;
            const double delta = cpaDelta<NC>(d, j, m, s.g);
            aC[j] = rho * x[j] * o.acceptor[j] * delta;
            bC[j] = rho * x[d] * o.donor[d] * delta;
            aSum += aC[j];
        }
        double donorX = 1.0 / (1.0 + aSum);
        double lower = 0.0, upper = 1.0;
        bool converged = false;
        const int maxIt = o.maxIterations < 64 ? o.maxIterations : 64;
        for (int it = 0; it < maxIt; ++it)
        {
            double sum = 0.0, slope = 0.0;
            for (int j = 0; j < NC; ++j)
            {
                if (o.acceptor[j] <= 0)
                    continue;
                const double denominator = 1.0 + bC[j] * donorX;
                sum += aC[j] / denominator;
                slope -= aC[j] * bC[j] / (denominator * denominator);
            }
            const double residual = donorX * (1.0 + sum) - 1.0;
            const double derivative = 1.0 + sum + donorX * slope;
            if (residual > 0.0)
                upper = donorX;
            else
                lower = donorX;
            if (fabs(residual) <= o.tolerance)
            {
                converged = true;
                break;
            }
            double candidate = donorX;
            if (isfinite(derivative) && fabs(derivative) > 1.0e-14)
                candidate = donorX - residual / derivative;
            if (!isfinite(candidate) || !(candidate > lower && candidate < upper))
            {
                const double midpoint = 0.5 * (lower + upper);
                candidate = donorX + (midpoint - donorX);
            }
            donorX = candidate;
        }
        if (!converged)
            return ERR_EOS;   // "CPA reduced association-site iteration did not converge."
        s.donorX[d] = donorX;
        for (int j = 0; j < NC; ++j)
            if (o.acceptor[j] > 0)
                s.acceptorX[j] = 1.0 / (1.0 + bC[j] * donorX);
    }
    else
    {
        // without donor sites nothing associates (every X stays 1); several
        // donor-bearing components take the general dense path (:1731-2030),
        // which is not carried here
        for (int i = 0; i < NC; ++i)
            if (o.donor[i] > 0)
                return ERR_NOT_PORTED;
    }
    s.bonded = 0.0;
    for (int i = 0; i < NC; ++i)
        s.bonded += x[i] * (o.donor[i] * (1.0 - s.donorX[i]) + o.acceptor[i] * (1.0 - s.acceptorX[i]));
    return ERR_NONE;
}

// cpaPressureAtDensityWithMix_ (cubic_eos.hpp:2050-2078).
template <int NC>
NZ_HD int cpaPressure(const FluidDev &F, double rho, double T, const double *x, const CpaMix<NC> &m, double &p)
{
    if (!(1.0 - m.b * rho > 0.0))
        return ERR_EOS;   // "CPA density exceeds the SRK co-volume limit."
    const double q = m.b * rho;
    double attraction = 1.0 + q;
    if (F.cpa.pengRobinson)
        attraction = (1.0 + (1.0 + kSqrtTwo) * q) * (1.0 + (1.0 - kSqrtTwo) * q);
    const double cubic = kGasConstant * T * rho / (1.0 - q) - m.a * rho * rho / attraction;
    CpaAssoc<NC> s;
    const int rc = cpaAssociation<NC>(F, rho, x, m, s);
    if (rc != ERR_NONE)
        return rc;
    const double factor = 1.0 + s.gPrimeOverG * m.b * rho / 4.0;
    const double association = -0.5 * kGasConstant * T * rho * factor * s.bonded;
    p = cubic + association;
    return ERR_NONE;
}

// cpaDensityRootValueWithMix_ (:2090-2178): bracket and bisection.
template <int NC>
NZ_HD int cpaDensityRootValue(const FluidDev &F, double P, double T, const double *x, bool liquid,
                              const CpaMix<NC> &m, double &rhoOut)
{
    const double b = m.b;
    if (!(b > 0.0))
        return ERR_EOS;
    const double rhoMax = 0.999999 / b;
    int rc = ERR_NONE;
    auto residual = [&](double rho) {
        double p = 0.0;
        const int e = cpaPressure<NC>(F, rho, T, x, m, p);
        if (e != ERR_NONE && rc == ERR_NONE)
            rc = e;
        return p - P;
    };
    double lo = 0.0, hi = 0.0, flo = -P, fhi = 0.0;
    if (!liquid)
    {
        const double start = 0.25 * P / (kGasConstant * T);
        hi = smin(rhoMax, smax(1.0, start));
        fhi = residual(hi);
        if (rc)
            return rc;
        while (fhi < 0.0 && hi < 0.999 * rhoMax)   // grows geometrically to rhoMax
        {
            lo = hi;
            flo = fhi;
            hi = smin(0.999999 * rhoMax, hi * 1.6 + 1.0);
            fhi = residual(hi);
            if (rc)
                return rc;
        }
    }
    else
    {
        hi = rhoMax;
        fhi = residual(hi);
        if (rc)
            return rc;
        lo = 0.82 * hi;
        flo = residual(lo);
        if (rc)
            return rc;
        for (int i = 0; i < 160 && flo > 0.0; ++i)
        {
            hi = lo;
            fhi = flo;
            lo *= 0.82;
            flo = residual(lo);
            if (rc)
                return rc;
        }
    }
    if (!(flo <= 0.0 && fhi >= 0.0))
        return ERR_EOS;   // "CPA could not bracket the requested density root."
    for (int it = 0; it < 100; ++it)
    {
        const double mid = 0.5 * (lo + hi);
        const double fm = residual(mid);
        if (rc)
            return rc;
        if (fm > 0.0)
        {
            hi = mid;
            fhi = fm;
        }
        else
        {
            lo = mid;
            flo = fm;
        }
        if (fabs(fm) <= 1.0e-10 * smax(P, 1.0) || (hi - lo) <= 1.0e-12 * smax(mid, 1.0))
            break;
    }
    rhoOut = 0.5 * (lo + hi);
    return ERR_NONE;
}

// cpaDensityRoot_ (:2191-2248) for scalar evaluations: the value root and its
// two implicit corrections with the scalar mixing state.
template <int NC>
NZ_HD int cpaDensityRoot(const FluidDev &F, double P, double T, const double *x, bool liquid, const CpaMix<NC> &m,
                         double &rhoOut)
{
    double rho = 0.0;
    int rc = cpaDensityRootValue<NC>(F, P, T, x, liquid, m, rho);
    if (rc != ERR_NONE)
        return rc;
    for (int correction = 0; correction < 2; ++correction)
    {
        const double h = smax(1.0e-4, fabs(rho) * 2.0e-6);
        const double lower = smax(1.0e-12, rho - h);
        const double upper = rho + h;
        double pLower = 0.0, pUpper = 0.0, pRho = 0.0;
        if ((rc = cpaPressure<NC>(F, lower, T, x, m, pLower)) != ERR_NONE)
            return rc;
        if ((rc = cpaPressure<NC>(F, upper, T, x, m, pUpper)) != ERR_NONE)
            return rc;
        const double derivative = (pUpper - pLower) / (upper - lower);
        if (!isfinite(derivative) || fabs(derivative) < 1.0e-12)
            return ERR_EOS;   // "CPA density root has a singular pressure derivative."
        if ((rc = cpaPressure<NC>(F, rho, T, x, m, pRho)) != ERR_NONE)
            return rc;
        const double r = pRho - P;
        rho -= r / derivative;
    }
    rhoOut = rho;
    return ERR_NONE;
}

// cpaAtDensity_ (:2250-2307): Z and the fugacity coefficients at density rho.
template <int NC>
NZ_HD int cpaAtDensity(const FluidDev &F, double P, double T, const double *x, double rho, double &Z, double *phi)
{
    const CpaDev &o = F.cpa;
    CpaMix<NC> m;
    cpaMixing<NC>(F, T, x, m);
    CpaAssoc<NC> s;
    int rc = cpaAssociation<NC>(F, rho, x, m, s);
    if (rc != ERR_NONE)
        return rc;
    const double q = m.b * rho;
    if (!(1.0 - q > 0.0))
        return ERR_EOS;   // "CPA fugacity requires b*rho < 1."
    Z = P / (rho * kGasConstant * T);
    double integral = log(1.0 + q);
    double derivative = 1.0 / (1.0 + q);
    if (o.pengRobinson)
    {
        const double first = 1.0 + (1.0 + kSqrtTwo) * q;
        const double second = 1.0 + (1.0 - kSqrtTwo) * q;
        integral = log(first / second) / (2.0 * kSqrtTwo);
        derivative = 1.0 / (first * second);
    }
    const double logZ = log(Z);
    for (int i = 0; i < NC; ++i)
    {
        const double bi = m.bi[i];
        double muCubic = -log(1.0 - q) + rho * bi / (1.0 - q);
        muCubic -= ((2.0 * m.Si[i] / m.b - m.a * bi / (m.b * m.b)) * integral + (m.a / m.b) * rho * bi * derivative) /
            (kGasConstant * T);
        double muAssociation = 0.0;
        if (o.donor[i] > 0)
            muAssociation += o.donor[i] * log(s.donorX[i]);
        if (o.acceptor[i] > 0)
            muAssociation += o.acceptor[i] * log(s.acceptorX[i]);
        const double dLnGdNi = s.gPrimeOverG * bi * rho / 4.0;
        muAssociation -= 0.5 * dLnGdNi * s.bonded;
        const double lnPhi = muCubic + muAssociation - logZ;
        phi[i] = exp(lnPhi);
    }
    return ERR_NONE;
}

// cpaPhaseResult_ with selectGibbsMinimum = false (:2309-2336).
template <int NC>
NZ_HD int cpaPhase(const FluidDev &F, double P, double T, const double *x, bool liquid, double &Z, double *phi)
{
    CpaMix<NC> m;
    cpaMixing<NC>(F, T, x, m);
    double rho = 0.0;
    const int rc = cpaDensityRoot<NC>(F, P, T, x, liquid, m, rho);
    if (rc != ERR_NONE)
        return rc;
    return cpaAtDensity<NC>(F, P, T, x, rho, Z, phi);
}

// ---------------------------------------------------------------------------
// The same phase evaluation over a differentiable scalar S (the Natural
// kernels' Dual, DualN<K> and Val): the reference templates cpaMixing_,
// cpaAssociationState_, cpaPressureAtDensityWithMix_, cpaDensityRoot_ and
// cpaAtDensity_ on its scalar, so the cell properties of a CPA fluid carry
// derivatives through the association solve and the density root.  The
// temperature-only parameters (ai, bi, aij and the association factors) are
// the scalar mixing state's -- at the isothermal reservoir temperature the
// reference takes them from its CPA temperature cache, with no derivatives --
// and only Si, a and b depend on the composition.  The root itself is found in
// FP64 (cpaDensityRootValue) and its derivatives injected by the reference's
// two implicit corrections.  Divisions follow the reference's scalar types
// (a scalar divided by a plain number multiplies by the reciprocal).

template <int NC, class S>
struct CpaMixT
{
    const CpaMix<NC> *t;   // temperature-only part (ai, bi, aij, factor, volume)
    S Si[NC];
    S a, b;
};

template <int NC, class S>
struct CpaAssocT
{
    S donorX[NC], acceptorX[NC];
    S g, gPrimeOverG, bonded;
};

template <int NC, class S>
NZ_HD void cpaMixingT(const CpaMix<NC> &t, const S *x, CpaMixT<NC, S> &m)
{
    m.t = &t;
    m.a = S(0.0);
    m.b = S(0.0);
    for (int i = 0; i < NC; ++i)
    {
        m.Si[i] = S(0.0);
        for (int j = 0; j < NC; ++j)
            m.Si[i] += x[j] * t.aij[i][j];
        m.a += x[i] * m.Si[i];
        m.b += x[i] * t.bi[i];
    }
}

template <class S>
NZ_HD void cpaRadialT(const FluidDev &F, const S &eta, S &g, S &gPrimeOverG)
{
    if (!F.cpa.carnahanStarling)
    {
        const S denominator = S(1.0) - 1.9 * eta;
        g = S(1.0) / denominator;
        gPrimeOverG = 1.9 * g;
        return;
    }
    const S oneMinusEta = S(1.0) - eta;
    g = (S(1.0) - 0.5 * eta) / (oneMinusEta * oneMinusEta * oneMinusEta);
    const S gPrime = (S(2.5) - eta) / (oneMinusEta * oneMinusEta * oneMinusEta * oneMinusEta);
    gPrimeOverG = gPrime / g;
}

template <int NC, class S>
NZ_HD S cpaDeltaT(int donor, int acceptor, const CpaMix<NC> &t, const S &g)
{
    const double temperatureFactor = t.factor[donor][acceptor];
    const double beta = t.volume[donor][acceptor];
    if (!(temperatureFactor > 0.0) || !(beta > 0.0))
        return S(0.0);
    const double bij = 0.5 * (t.bi[donor] + t.bi[acceptor]);
    return g * temperatureFactor * bij * beta;
}

template <int NC, class S>
NZ_HD int cpaAssociationT(const FluidDev &F, const S &rho, const S *x, const CpaMixT<NC, S> &m, CpaAssocT<NC, S> &s)
{
    const CpaDev &o = F.cpa;
    const CpaMix<NC> &t = *m.t;
    for (int i = 0; i < NC; ++i)
    {
        s.donorX[i] = S(1.0);
        s.acceptorX[i] = S(1.0);
    }
    const S eta = m.b * rho / 4.0;
    cpaRadialT<S>(F, eta, s.g, s.gPrimeOverG);
    if (o.symmetric >= 0)
    {
        const int k = o.symmetric;
        const int sites = o.donor[k];
        const S delta = cpaDeltaT<NC, S>(k, k, t, s.g);
        const S A = rho * x[k] * static_cast<double>(sites) * delta;
        const S X = S(2.0) / (S(1.0) + sqrt(S(1.0) + S(4.0) * A));
        s.donorX[k] = X;
        s.acceptorX[k] = X;
    }
    else if (o.singleDonor >= 0)
    {
        const int d = o.singleDonor;
        S aC[NC], bC[NC];
        S aSum = S(0.0);
        for (int j = 0; j < NC; ++j)
        {
            aC[j] = S(0.0);
            bC[j] = S(0.0);
            if (o.acceptor[j] <= 0)
                continue;
            const S delta = cpaDeltaT<NC, S>(d, j, t, s.g);
            aC[j] = rho * x[j] * o.acceptor[j] * delta;
            bC[j] = rho * x[d] * o.donor[d] * delta;
            aSum += aC[j];
        }
        S donorX = S(1.0) / (S(1.0) + aSum);
        double lower = 0.0, upper = 1.0;
        bool converged = false;
        const int maxIt = o.maxIterations < 64 ? o.maxIterations : 64;
        for (int it = 0; it < maxIt; ++it)
        {
            S sum = S(0.0), slope = S(0.0);
            for (int j = 0; j < NC; ++j)
            {
                if (o.acceptor[j] <= 0)
                    continue;
                const S denominator = S(1.0) + bC[j] * donorX;
                sum += aC[j] / denominator;
                slope -= aC[j] * bC[j] / (denominator * denominator);
            }
            const S residual = donorX * (S(1.0) + sum) - 1.0;
            const S derivative = S(1.0) + sum + donorX * slope;
            const double residualValue = val(residual);
            const double donorValue = val(donorX);
            if (residualValue > 0.0)
                upper = donorValue;
            else
                lower = donorValue;
            if (fabs(residualValue) <= o.tolerance)
            {
                converged = true;
                break;
            }
            const double derivativeValue = val(derivative);
            S candidate = donorX;
            if (isfinite(derivativeValue) && fabs(derivativeValue) > 1.0e-14)
                candidate = donorX - residual / derivative;
            const double candidateValue = val(candidate);
            if (!isfinite(candidateValue) || !(candidateValue > lower && candidateValue < upper))
            {
                const double midpoint = 0.5 * (lower + upper);
                candidate = donorX + (midpoint - donorValue);
            }
            donorX = candidate;
        }
        if (!converged)
            return ERR_EOS;
        s.donorX[d] = donorX;
        for (int j = 0; j < NC; ++j)
            if (o.acceptor[j] > 0)
                s.acceptorX[j] = S(1.0) / (S(1.0) + bC[j] * donorX);
    }
    else
    {
        for (int i = 0; i < NC; ++i)
            if (o.donor[i] > 0)
                return ERR_NOT_PORTED;
    }
    s.bonded = S(0.0);
    for (int i = 0; i < NC; ++i)
        s.bonded += x[i] * (o.donor[i] * (S(1.0) - s.donorX[i]) + o.acceptor[i] * (S(1.0) - s.acceptorX[i]));
    return ERR_NONE;
}

template <int NC, class S>
NZ_HD int cpaPressureT(const FluidDev &F, const S &rho, double T, const S *x, const CpaMixT<NC, S> &m, S &p)
{
    if (!(val(S(1.0) - m.b * rho) > 0.0))
        return ERR_EOS;
    const S q = m.b * rho;
    S attraction = S(1.0) + q;
    if (F.cpa.pengRobinson)
        attraction = (S(1.0) + (1.0 + kSqrtTwo) * q) * (S(1.0) + (1.0 - kSqrtTwo) * q);
    const S cubic = S(kGasConstant * T) * rho / (S(1.0) - q) - m.a * rho * rho / attraction;
    CpaAssocT<NC, S> s;
    const int rc = cpaAssociationT<NC, S>(F, rho, x, m, s);
    if (rc != ERR_NONE)
        return rc;
    const S factor = S(1.0) + s.gPrimeOverG * m.b * rho / 4.0;
    const S association = S(-0.5 * kGasConstant * T) * rho * factor * s.bonded;
    p = cubic + association;
    return ERR_NONE;
}

template <int NC, class S>
NZ_HD int cpaAtDensityT(const FluidDev &F, const S &P, double T, const S *x, const S &rho, const CpaMix<NC> &t,
                        S &Z, S *phi)
{
    const CpaDev &o = F.cpa;
    CpaMixT<NC, S> m;
    cpaMixingT<NC, S>(t, x, m);
    CpaAssocT<NC, S> s;
    const int rc = cpaAssociationT<NC, S>(F, rho, x, m, s);
    if (rc != ERR_NONE)
        return rc;
    const S q = m.b * rho;
    if (!(val(S(1.0) - q) > 0.0))
        return ERR_EOS;
    const S RT = S(kGasConstant * T);
    Z = P / (rho * kGasConstant * S(T));
    S integral = log(S(1.0) + q);
    S derivative = S(1.0) / (S(1.0) + q);
    if (o.pengRobinson)
    {
        const S first = S(1.0) + (1.0 + kSqrtTwo) * q;
        const S second = S(1.0) + (1.0 - kSqrtTwo) * q;
        integral = log(first / second) / (2.0 * kSqrtTwo);
        derivative = S(1.0) / (first * second);
    }
    const S logZ = log(Z);
    for (int i = 0; i < NC; ++i)
    {
        const double bi = t.bi[i];
        S muCubic = -log(S(1.0) - q) + rho * bi / (S(1.0) - q);
        muCubic -= ((2.0 * m.Si[i] / m.b - m.a * bi / (m.b * m.b)) * integral + (m.a / m.b) * rho * bi * derivative) /
            RT;
        S muAssociation = S(0.0);
        if (o.donor[i] > 0)
            muAssociation += o.donor[i] * log(s.donorX[i]);
        if (o.acceptor[i] > 0)
            muAssociation += o.acceptor[i] * log(s.acceptorX[i]);
        const S dLnGdNi = s.gPrimeOverG * bi * rho / 4.0;
        muAssociation -= 0.5 * dLnGdNi * s.bonded;
        const S lnPhi = muCubic + muAssociation - logZ;
        phi[i] = exp(lnPhi);
    }
    return ERR_NONE;
}

// cpaPhaseResult_ (:2309-2336) over S: Z and the fugacity coefficients.
template <int NC, class S>
NZ_HD int cpaPhaseT(const FluidDev &F, const S &P, double T, const S *x, bool liquid, S &Z, S *phi)
{
    double xv[NC];
    for (int i = 0; i < NC; ++i)
        xv[i] = val(x[i]);
    const double pValue = val(P);
    CpaMix<NC> t;
    cpaMixing<NC>(F, T, xv, t);
    double root = 0.0;
    int rc = cpaDensityRootValue<NC>(F, pValue, T, xv, liquid, t, root);
    if (rc != ERR_NONE)
        return rc;
    S rho = S(root);
    CpaMixT<NC, S> m;
    cpaMixingT<NC, S>(t, x, m);
    for (int correction = 0; correction < 2; ++correction)
    {
        const double rhoValue = val(rho);
        const double h = smax(1.0e-4, fabs(rhoValue) * 2.0e-6);
        const double lower = smax(1.0e-12, rhoValue - h);
        const double upper = rhoValue + h;
        double pLower = 0.0, pUpper = 0.0;
        if ((rc = cpaPressure<NC>(F, lower, T, xv, t, pLower)) != ERR_NONE)
            return rc;
        if ((rc = cpaPressure<NC>(F, upper, T, xv, t, pUpper)) != ERR_NONE)
            return rc;
        const double derivative = (pUpper - pLower) / (upper - lower);
        if (!isfinite(derivative) || fabs(derivative) < 1.0e-12)
            return ERR_EOS;
        S pRho;
        if ((rc = cpaPressureT<NC, S>(F, rho, T, x, m, pRho)) != ERR_NONE)
            return rc;
        const S residual = pRho - P;
        rho = rho - residual / derivative;
    }
    return cpaAtDensityT<NC, S>(F, P, T, x, rho, t, Z, phi);
}

} // namespace nz
