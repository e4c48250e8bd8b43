// eos.cuh -- device cubic equation of state (PR / PR78 / Soreide-Whitson).
//
// Restates, for one thread and one (P, T), the reference's
// CubicEquationOfState (models/include/natural/thermo/cubic_eos.hpp):
//   mixingParameters  :581-650      phaseMixing     :666-692
//   cubicCoefficients :696-705      solveCubic      :707-756
//   liquidRoot        :760-780      vaporRoot       :783-803
//   fugacityAtRoot    :902-934      molarDensity    :481-550 (no translation)
// and SoreideWhitsonCorrelations (soreide_whitson.hpp:25-166).
// The operation order of every expression follows the reference so that the
// FP64 path agrees with it to rounding; std::max/min/clamp NaN semantics are
// kept (smax/smin/sclamp below), they matter for the reference's guards.
#pragma once

#include <cstdint>
#include <math.h>

// Device code is CUDA; the same headers also compile as plain C++ so that a
// host build can be used to step through a point when debugging.
#ifdef __CUDACC__
#define NZ_HD __device__
#define NZ_HDI __device__ __forceinline__
#define NZ_HDN __device__ __noinline__
#define NZ_BOTH __host__ __device__ inline
#else
#define NZ_BOTH inline
#include <cmath>
#include <cstring>
using std::isfinite;
#define NZ_HD
#define NZ_HDI inline
#define NZ_HDN __attribute__((noinline))
#endif

namespace nz
{

NZ_HDI double nzNan()
{
#ifdef __CUDACC__
    return __longlong_as_double(0x7ff8000000000000LL);
#else
    return std::nan("");
#endif
}
NZ_HDI double nzInf()
{
#ifdef __CUDACC__
    return __longlong_as_double(0x7ff0000000000000LL);
#else
    return HUGE_VAL;
#endif
}
NZ_HDI int imin(int a, int b) { return a < b ? a : b; }
NZ_HDI int imax(int a, int b) { return a < b ? b : a; }

constexpr double kGasConstant = 8.31446261815324;   // common/units.hpp
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kBar = 100000.0;
constexpr int kMaxNc = 8;

// Phase slots / thermodynamic roles (phase_behavior.hpp:15-20)
constexpr int OIL = 0;
constexpr int GAS = 1;
constexpr int WATER = 2;
constexpr uint8_t OIL_BIT = 1, GAS_BIT = 2, WATER_BIT = 4, ALL_BITS = 7;

constexpr int EOS_PR = 0;
constexpr int EOS_SW = 1;
constexpr int EOS_CPA = 2;

// Error codes a thread can raise where the reference throws.
constexpr int ERR_NONE = 0;
constexpr int ERR_BAD_INPUT = 2;   // std::invalid_argument in the reference
constexpr int ERR_EOS = 3;         // std::runtime_error in the reference
constexpr int ERR_NOT_PORTED = 4;

// std::max / std::min / std::clamp with the same NaN behaviour as libstdc++.
NZ_HDI double smax(double a, double b) { return (a < b) ? b : a; }
NZ_HDI double smin(double a, double b) { return (b < a) ? b : a; }
NZ_HDI double smax3(double a, double b, double c)
{
    double r = a;
    if (r < b) r = b;
    if (r < c) r = c;
    return r;
}
NZ_HDI double sclamp(double v, double lo, double hi)
{
    return (v < lo) ? lo : ((hi < v) ? hi : v);
}
NZ_HDI int bitOf(int slot) { return 1 << slot; }
NZ_HDI int popcount3(uint8_t b)
{
    return (b & 1) + ((b >> 1) & 1) + ((b >> 2) & 1);
}

struct FlashOpts
{
    int maxIterations;
    int maxRr;
    int maxStability;
    int stabilitySsi;
    int stabilityNewton;
    int twoSsi;
    int twoNewton;
    int threeSsi;
    int threeNewton;
    double fugacityTol;
    double rrTol;
    double stabilityTol;
    double betaTol;
    double coincidentTol;
    double floor;
    double logKLimit;
    double fdStep;
};

// Cubic-plus-association parameters (CubicEquationOfState::CubicPlusAssociationOptions,
// cubic_eos.hpp:117-136), with the association scheme classified once on the host.
struct CpaDev
{
    double a0[kMaxNc], b[kMaxNc], c1[kMaxNc];
    double epsilon[kMaxNc], beta[kMaxNc];
    int donor[kMaxNc], acceptor[kMaxNc];
    double crossEpsilon[kMaxNc * kMaxNc], crossBeta[kMaxNc * kMaxNc];
    int pengRobinson;        // physical term: 1 Peng-Robinson, 0 Soave-Redlich-Kwong
    int carnahanStarling;    // radial distribution: 1 Carnahan-Starling, 0 simplified
    int maxIterations;
    double tolerance;
    double damping;
    int symmetric;           // the only associating component, with equal donor/acceptor sites, else -1
    int singleDonor;         // the only donor-bearing component, else -1
};

// Fluid constants as kernels see them (by value, __grid_constant__).
struct FluidDev
{
    int nc;
    int eosModel;
    int eosType;
    int water;
    double omegaA, omegaB, m1, m2;
    double minComposition;
    double tc[kMaxNc], pc[kMaxNc], vc[kMaxNc], omega[kMaxNc], mw[kMaxNc];
    double kij[kMaxNc * kMaxNc];
    double salinity;
    int swKind[kMaxNc];
    double swValue[kMaxNc];
    FlashOpts opt;
    CpaDev cpa;
    // Iterations a lane-refill loop of the staged kernels may run before it
    // gives up and sets the batch's guard word (a self-check, not a
    // convergence limit: the solves end far earlier).
    long long spinLimit;
};

template <int NC>
struct MixParams
{
    double A[NC][NC];
    double B[NC];
};

template <int NC>
struct PhaseMix
{
    double S[NC];
    double A;
    double B;
};

// ---- Soreide-Whitson correlations (soreide_whitson.hpp) -------------------
NZ_HDI double swWaterAlpha(double T, double tcw, double salinity)
{
    const double tr = T / tcw;
    const double saltFactor = 1.0 - 0.0103 * pow(salinity, 1.1);
    const double sqrtAlpha = 1.0 + 0.4530 * (1.0 - tr * saltFactor)
        + 0.0034 * (pow(tr, -3.0) - 1.0);
    return sqrtAlpha * sqrtAlpha;
}

NZ_HDI double swHydrocarbonBip(double T, double tc, double omega, double s)
{
    const double tr = T / tc;
    const double a0 = 1.1120 - 1.7369 * pow(omega, -0.1);
    const double a1 = 1.1001 + 0.8360 * omega;
    const double a2 = -0.15742 - 1.0988 * omega;
    const double alpha0 = 0.017407, alpha1 = 0.033516, alpha2 = 0.011478;
    return a0 * (1.0 + alpha0 * s) + a1 * tr * (1.0 + alpha1 * s)
        + a2 * tr * tr * (1.0 + alpha2 * s);
}

NZ_HDI double swCo2Bip(double T, double tc, double s)
{
    const double tr = T / tc;
    return -0.31092 * (1.0 + 0.15587 * pow(s, 0.7505))
        + 0.2358 * (1.0 + 0.17837 * pow(s, 0.979)) * tr
        - 21.2566 * exp(-6.7222 * tr - s);
}

NZ_HDI double swCo2BipChabab(double T, double s)
{
    const double tr = T / 304.13;
    const double a = 0.43575155, b = -0.05766906744, c = 0.00826464849;
    const double d = 0.00129539193, e = -0.0016698848, f = -0.47866096;
    return tr * (a + b * tr + c * tr * s) + s * s * (d + e * tr) + f;
}

// soreideWhitsonAqueousBip_ (cubic_eos.hpp:2389-2404)
NZ_HDI double swAqueousBip(const FluidDev &F, int i, int j, double T, double s)
{
    const int w = F.water;
    if (i != w && j != w)
        return F.kij[i * kMaxNc + j];
    if (i == w && j == w)
        return 0.0;
    const int other = (i == w) ? j : i;
    switch (F.swKind[other])
    {
    case 1: return F.swValue[other];
    case 2: return swCo2Bip(T, F.tc[other], s);
    case 3: return swHydrocarbonBip(T, F.tc[other], F.omega[other], s);
    case 4: return swCo2BipChabab(T, s);
    default: return F.kij[i * kMaxNc + j];
    }
}

// mixingParameters(P, T, role) (cubic_eos.hpp:581-650)
template <int NC>
NZ_HD void mixingParameters(const FluidDev &F, double P, double T, double salinity,
                                 bool aqueousRole, MixParams<NC> &out)
{
    double sqrtAi[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i)
    {
        const double pr = P / F.pc[i];
        const double tr = T / F.tc[i];
        double alpha;
        if (F.eosModel == EOS_SW && i == F.water)
        {
            alpha = swWaterAlpha(T, F.tc[i], salinity);
        }
        else
        {
            const double omega = F.omega[i];
            double m = 0.37464 + 1.54226 * omega - 0.26992 * omega * omega;
            if (F.eosType == 5 && omega > 0.49)
                m = 0.379642 + 1.48503 * omega - 0.164423 * omega * omega
                    + 0.016666 * omega * omega * omega;
            const double alphaRoot = 1.0 + m * (1.0 - sqrt(tr));
            alpha = alphaRoot * alphaRoot;
        }
        const double reducedA = F.omegaA * alpha * pr / (tr * tr);
        sqrtAi[i] = sqrt(reducedA);
        out.B[i] = F.omegaB * pr / tr;
    }
    const bool swAq = F.eosModel == EOS_SW && aqueousRole;
#pragma unroll
    for (int i = 0; i < NC; ++i)
    {
#pragma unroll
        for (int j = i; j < NC; ++j)
        {
            double kij = F.kij[i * kMaxNc + j];
            if (swAq)
                kij = swAqueousBip(F, i, j, T, salinity);
            const double aij = sqrtAi[i] * sqrtAi[j] * (1.0 - kij);
            out.A[i][j] = aij;
            out.A[j][i] = aij;
        }
    }
}

// phaseMixing (cubic_eos.hpp:666-692)
template <int NC>
NZ_HDI void phaseMixing(const double *x, const MixParams<NC> &p, PhaseMix<NC> &m)
{
    m.A = 0.0;
    m.B = 0.0;
#pragma unroll
    for (int i = 0; i < NC; ++i)
    {
        double si = 0.0;
#pragma unroll
        for (int j = 0; j < NC; ++j)
            si += x[j] * p.A[i][j];
        m.S[i] = si;
        m.B += x[i] * p.B[i];
    }
#pragma unroll
    for (int i = 0; i < NC; ++i)
        m.A += x[i] * m.S[i];
}

// solveCubic + liquid/vapour root choice (cubic_eos.hpp:696-803).
// Returns the selected root or NaN (the reference throws) when none has Z > B.
NZ_HDI double selectCubicRoot(double A, double B, double m1, double m2, bool vapour)
{
    const double e0 = -(A * B + m1 * m2 * B * B * (B + 1.0));
    const double e1 = A - (m1 + m2 - m1 * m2) * B * B - (m1 + m2) * B;
    const double e2 = (m1 + m2 - 1.0) * B - 1.0;
    const double a = e2, b = e1, c = e0;
    const double Q = (a * a - 3.0 * b) / 9.0;
    const double R = (2.0 * a * a * a - 9.0 * a * b + 27.0 * c) / 54.0;
    const double disc = R * R - Q * Q * Q;
    const double nan = nzNan();
    double r0 = nan, r1 = nan, r2 = nan;
    if (disc < 0.0)
    {
        double arg = R / sqrt(Q * Q * Q);
        if (arg > 1.0)
            arg = 1.0;
        else if (arg < -1.0)
            arg = -1.0;
        const double theta = acos(arg);
        const double sq = sqrt(Q);
        r0 = -2.0 * sq * cos(theta / 3.0) - a / 3.0;
        r1 = -2.0 * sq * cos((theta + 2.0 * kPi) / 3.0) - a / 3.0;
        r2 = -2.0 * sq * cos((theta - 2.0 * kPi) / 3.0) - a / 3.0;
    }
    else
    {
        double S;
        if (R > 0.0)
            S = -pow(fabs(R) + sqrt(disc), 1.0 / 3.0);
        else
            S = pow(fabs(R) + sqrt(disc), 1.0 / 3.0);
        double Tt = 0.0;
        if (fabs(S) > 0.0)
            Tt = Q / S;
        r0 = S + Tt - a / 3.0;
    }
    if (isfinite(r0) && r0 <= 0.0) r0 = nan;
    if (isfinite(r1) && r1 <= 0.0) r1 = nan;
    if (isfinite(r2) && r2 <= 0.0) r2 = nan;
    bool found = false;
    double best = nan;
    const double roots[3] = {r0, r1, r2};
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        const double z = roots[k];
        if (!isfinite(z) || !(z > B))
            continue;
        if (!found || (vapour ? (z > best) : (z < best)))
        {
            best = z;
            found = true;
        }
    }
    return best;
}

// fugacityAtRoot (cubic_eos.hpp:902-934): phi_i = exp(ln phi_i).
// Returns false where the reference throws.
template <int NC>
NZ_HDI bool fugacityCoefficients(const double *x, const MixParams<NC> &p,
                                                     const PhaseMix<NC> &m, double Z,
                                                     double m1, double m2, double *phi)
{
    if (!(m.B > 0.0) || !(m.A > 0.0))
        return false;
    if (!(Z - m.B > 0.0))
        return false;
    const double commonA = -log(Z - m.B);
    const double logRatio = log((Z + m2 * m.B) / (Z + m1 * m.B));
    const double commonB = logRatio * m.A / ((m1 - m2) * m.B);
    const double commonC = (Z - 1.0) / m.B;
#pragma unroll
    for (int i = 0; i < NC; ++i)
    {
        const double lnPhi = commonA + commonB * (2.0 * m.S[i] / m.A - p.B[i] / m.B)
            + p.B[i] * commonC;
        phi[i] = exp(lnPhi);
    }
    (void)x;
    return true;
}

// ln phi_i of one phase with the mixing sums and the fugacity expression in
// FP32 and the cubic root chosen in FP64 (the mixed-precision form's
// successive-substitution evaluations).  False when the FP32 evaluation has no
// admissible root or a non-finite term; the caller then evaluates in FP64.
template <int NC>
NZ_HDI bool lnPhiMixed(const double *x, const MixParams<NC> &p, double m1, double m2, bool vapour,
                       double *lnphi)
{
    float xf[NC], S[NC];
    float A = 0.0f, B = 0.0f;
#pragma unroll
    for (int i = 0; i < NC; ++i)
        xf[i] = float(x[i]);
#pragma unroll
    for (int i = 0; i < NC; ++i)
    {
        float si = 0.0f;
#pragma unroll
        for (int j = 0; j < NC; ++j)
            si += xf[j] * float(p.A[i][j]);
        S[i] = si;
        B += xf[i] * float(p.B[i]);
    }
#pragma unroll
    for (int i = 0; i < NC; ++i)
        A += xf[i] * S[i];
    if (!(B > 0.0f) || !(A > 0.0f))
        return false;
    const double Z = selectCubicRoot(double(A), double(B), m1, m2, vapour);
    if (!isfinite(Z) || !(Z - double(B) > 0.0))
        return false;
    const float z = float(Z), m1f = float(m1), m2f = float(m2);
    const float commonA = -logf(z - B);
    const float commonB = logf((z + m2f * B) / (z + m1f * B)) * A / ((m1f - m2f) * B);
    const float commonC = (z - 1.0f) / B;
    bool ok = isfinite(commonA) && isfinite(commonB) && isfinite(commonC);
#pragma unroll
    for (int i = 0; i < NC; ++i)
    {
        const float l = commonA + commonB * (2.0f * S[i] / A - float(p.B[i]) / B) + float(p.B[i]) * commonC;
        ok = ok && isfinite(l);
        lnphi[i] = double(l);
    }
    return ok;
}

// molarDensity without volume translation (cubic_eos.hpp:511-523)
NZ_HDI double molarDensity(double P, double T, double Z)
{
    return P / (kGasConstant * T * Z);
}

} // namespace nz
