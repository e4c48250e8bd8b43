/*
 * nz_oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C restatement of the
 * reference's thermodynamic building blocks, used by tests/ as an
 * independent checker next to oracle/_ref (the reference's own code).
 * Nothing in the product links or calls it.
 *
 * Restated (MPMC_SCW paths):
 *   mixing parameters   models/include/natural/thermo/cubic_eos.hpp:581-650
 *   SW water alpha and aqueous BIPs   thermo/soreide_whitson.hpp:25-134
 *   phase mixing        cubic_eos.hpp:666-692
 *   cubic roots         cubic_eos.hpp:696-803
 *   ln phi              cubic_eos.hpp:902-934
 *   two-phase RR        thermo/detail/three_phase_flash_nonlinear.inc:129-187
 *   three-phase RR      three_phase_flash_nonlinear.inc:8-96
 *   Wilson K            three_phase_flash_core.inc:152-165
 *   TPD residual        three_phase_flash_stability.inc:157-204
 *   LBC viscosity       models/include/natural/properties/compositional_properties.hpp:106-150
 * Pinned by tests/test_restatement.py against the reference's known answers
 * (test/src/unit/natural_core_test.cpp:83-125) and against oracle/_ref.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#include "../include/nonenone_b200.h"

#define R_GAS 8.31446261815324
#define PI 3.141592653589793238462643383279502884
#define MAXNC NZ_MAX_NC

static double sw_water_alpha(double T, double tcw, double s)
{
    const double tr = T / tcw;
    const double salt = 1.0 - 0.0103 * pow(s, 1.1);
    const double sa = 1.0 + 0.4530 * (1.0 - tr * salt) + 0.0034 * (pow(tr, -3.0) - 1.0);
    return sa * sa;
}

static double sw_aqueous_bip(const nz_fluid_desc *f, int i, int j, double T, double s)
{
    const int w = f->water_component;
    if (i != w && j != w)
        return f->kij[i * MAXNC + j];
    if (i == w && j == w)
        return 0.0;
    const int o = i == w ? j : i;
    const double tr = T / f->tc[o];
    switch (f->sw_bip_kind[o])
    {
    case NZ_SW_BIP_CONSTANT:
        return f->sw_bip_value[o];
    case NZ_SW_BIP_CO2:
        return -0.31092 * (1.0 + 0.15587 * pow(s, 0.7505))
            + 0.2358 * (1.0 + 0.17837 * pow(s, 0.979)) * tr
            - 21.2566 * exp(-6.7222 * tr - s);
    case NZ_SW_BIP_HYDROCARBON: {
        const double om = f->acentric[o];
        const double a0 = 1.1120 - 1.7369 * pow(om, -0.1);
        const double a1 = 1.1001 + 0.8360 * om;
        const double a2 = -0.15742 - 1.0988 * om;
        return a0 * (1.0 + 0.017407 * s) + a1 * tr * (1.0 + 0.033516 * s)
            + a2 * tr * tr * (1.0 + 0.011478 * s);
    }
    case NZ_SW_BIP_CO2_CHABAB: {
        const double t = T / 304.13;
        return t * (0.43575155 - 0.05766906744 * t + 0.00826464849 * t * s)
            + s * s * (0.00129539193 - 0.0016698848 * t) - 0.47866096;
    }
    default:
        return f->kij[i * MAXNC + j];
    }
}

/* A_ij (row-major MAXNC x MAXNC) and B_i at (P, T) for a role. */
void nzo_mixing(const nz_fluid_desc *f, double P, double T, double s, int role,
                double *A, double *B)
{
    const int n = f->nc;
    double sq[MAXNC];
    for (int i = 0; i < n; ++i)
    {
        const double pr = P / f->pc[i];
        const double tr = T / f->tc[i];
        double alpha;
        if (f->eos_model == NZ_EOS_SW && i == f->water_component)
        {
            alpha = sw_water_alpha(T, f->tc[i], s);
        }
        else
        {
            const double om = f->acentric[i];
            double m = 0.37464 + 1.54226 * om - 0.26992 * om * om;
            if (f->eos_type == 5 && om > 0.49)
                m = 0.379642 + 1.48503 * om - 0.164423 * om * om + 0.016666 * om * om * om;
            const double ar = 1.0 + m * (1.0 - sqrt(tr));
            alpha = ar * ar;
        }
        sq[i] = sqrt(f->omega_a * alpha * pr / (tr * tr));
        B[i] = f->omega_b * pr / tr;
    }
    const int aq = f->eos_model == NZ_EOS_SW && role == 2;
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j)
        {
            const double k = aq ? sw_aqueous_bip(f, i, j, T, s) : f->kij[i * MAXNC + j];
            const double a = sq[i] * sq[j] * (1.0 - k);
            A[i * MAXNC + j] = a;
            A[j * MAXNC + i] = a;
        }
}

/* Liquid (vapour=0) or vapour root with Z > B; NaN when none. */
double nzo_root(double A, double B, double m1, double m2, int vapour)
{
    const double e0 = -(A * B + m1 * m2 * B * B * (B + 1.0));
    const double e1 = A - (m1 + m2 - m1 * m2) * B * B - (m1 + m2) * B;
    const double e2 = (m1 + m2 - 1.0) * B - 1.0;
    const double Q = (e2 * e2 - 3.0 * e1) / 9.0;
    const double R = (2.0 * e2 * e2 * e2 - 9.0 * e2 * e1 + 27.0 * e0) / 54.0;
    const double d = R * R - Q * Q * Q;
    double r[3] = {NAN, NAN, NAN};
    if (d < 0.0)
    {
        double a = R / sqrt(Q * Q * Q);
        if (a > 1.0) a = 1.0;
        else if (a < -1.0) a = -1.0;
        const double th = acos(a);
        r[0] = -2.0 * sqrt(Q) * cos(th / 3.0) - e2 / 3.0;
        r[1] = -2.0 * sqrt(Q) * cos((th + 2.0 * PI) / 3.0) - e2 / 3.0;
        r[2] = -2.0 * sqrt(Q) * cos((th - 2.0 * PI) / 3.0) - e2 / 3.0;
    }
    else
    {
        const double S = (R > 0.0 ? -1.0 : 1.0) * pow(fabs(R) + sqrt(d), 1.0 / 3.0);
        const double Tt = fabs(S) > 0.0 ? Q / S : 0.0;
        r[0] = S + Tt - e2 / 3.0;
    }
    double best = NAN;
    int found = 0;
    for (int k = 0; k < 3; ++k)
    {
        const double z = r[k];
        if (!isfinite(z) || z <= 0.0 || !(z > B))
            continue;
        if (!found || (vapour ? z > best : z < best))
        {
            best = z;
            found = 1;
        }
    }
    return best;
}

/* One EOS phase evaluation: returns Z, fills lnphi[nc]; NaN when no root. */
double nzo_phase(const nz_fluid_desc *f, double P, double T, double s, const double *x,
                 int role, double *lnphi)
{
    const int n = f->nc;
    double A[MAXNC * MAXNC], B[MAXNC], S[MAXNC];
    nzo_mixing(f, P, T, s, role, A, B);
    double Am = 0.0, Bm = 0.0;
    for (int i = 0; i < n; ++i)
    {
        double si = 0.0;
        for (int j = 0; j < n; ++j)
            si += x[j] * A[i * MAXNC + j];
        S[i] = si;
        Bm += x[i] * B[i];
    }
    for (int i = 0; i < n; ++i)
        Am += x[i] * S[i];
    const double Z = nzo_root(Am, Bm, f->m1, f->m2, role == 1);
    if (!isfinite(Z) || !(Bm > 0.0) || !(Am > 0.0) || !(Z - Bm > 0.0))
    {
        for (int i = 0; i < n; ++i)
            lnphi[i] = NAN;
        return NAN;
    }
    const double ca = -log(Z - Bm);
    const double cb = log((Z + f->m2 * Bm) / (Z + f->m1 * Bm)) * Am / ((f->m1 - f->m2) * Bm);
    const double cc = (Z - 1.0) / Bm;
    for (int i = 0; i < n; ++i)
        lnphi[i] = ca + cb * (2.0 * S[i] / Am - B[i] / Bm) + B[i] * cc;
    return Z;
}

/* Two-phase RR on beta of the second phase; returns 1 on convergence. */
int nzo_rr2(int n, const double *z, const double *K, double init, double tol, int maxit,
            double *beta)
{
    double f0 = 0.0, f1 = 0.0;
    for (int i = 0; i < n; ++i)
    {
        f0 += z[i] * (K[i] - 1.0);
        f1 += z[i] * (K[i] - 1.0) / K[i];
    }
    if (!isfinite(f0) || !isfinite(f1))
        return 0;
    if (f0 <= 0.0) { *beta = 0.0; return 1; }
    if (f1 >= 0.0) { *beta = 1.0; return 1; }
    double lo = 0.0, hi = 1.0, b = init < 0.0 ? 0.0 : (init > 1.0 ? 1.0 : init);
    for (int it = 0; it < maxit; ++it)
    {
        double f = 0.0, df = 0.0;
        for (int i = 0; i < n; ++i)
        {
            const double a = K[i] - 1.0;
            const double D = (1.0 - b) + b * K[i];
            if (!(D > 1e-300))
                return 0;
            f += z[i] * a / D;
            df -= z[i] * a * a / (D * D);
        }
        if (fabs(f) < tol) { *beta = b; return 1; }
        if (f > 0.0) lo = b; else hi = b;
        double c = fabs(df) > 1e-24 ? b - f / df : b;
        if (!isfinite(c) || c <= lo || c >= hi)
            c = 0.5 * (lo + hi);
        b = c;
    }
    return 0;
}

/* Three-phase RR residual max norm at (bg, bw); inf outside the simplex. */
double nzo_rr3_norm(int n, const double *z, const double *kg, const double *kw, double bg, double bw)
{
    if (!(bg > 0.0) || !(bw > 0.0) || !(bg + bw < 1.0))
        return INFINITY;
    double fg = 0.0, fw = 0.0;
    for (int i = 0; i < n; ++i)
    {
        const double D = (1.0 - bg - bw) + bg * kg[i] + bw * kw[i];
        if (!(D > 1e-12))
            return INFINITY;
        fg += z[i] * (kg[i] - 1.0) / D;
        fw += z[i] * (kw[i] - 1.0) / D;
    }
    return fabs(fg) > fabs(fw) ? fabs(fg) : fabs(fw);
}

void nzo_wilson(const nz_fluid_desc *f, double P, double T, double *K)
{
    for (int i = 0; i < f->nc; ++i)
    {
        const double k = exp(log(f->pc[i] / P) + 5.373 * (1.0 + f->acentric[i]) * (1.0 - f->tc[i] / T));
        K[i] = k < 1e-30 ? 1e-30 : (k > 1e30 ? 1e30 : k);
    }
}

/* TPD stationarity residual max |ln W_i + ln phi_i(w) - ln x_ref,i - ln phi_ref,i|
 * for a trial W (not normalised) in the candidate role. */
double nzo_tpd_residual(const nz_fluid_desc *f, double P, double T, double s, const double *W,
                        int role, const double *xref, int refRole, double *trialSum)
{
    const int n = f->nc;
    double w[MAXNC], lw[MAXNC], lr[MAXNC], sum = 0.0;
    for (int i = 0; i < n; ++i)
        sum += W[i];
    for (int i = 0; i < n; ++i)
        w[i] = W[i] / sum;
    *trialSum = sum;
    if (!isfinite(nzo_phase(f, P, T, s, w, role, lw)) || !isfinite(nzo_phase(f, P, T, s, xref, refRole, lr)))
        return NAN;
    double r = 0.0;
    for (int i = 0; i < n; ++i)
    {
        const double xi = xref[i] > 1e-30 ? xref[i] : 1e-30;
        const double d = fabs(log(W[i]) + lw[i] - log(xi) - lr[i]);
        if (d > r)
            r = d;
    }
    return r;
}

/* LBC viscosity [Pa s] at molar density rho [mol/m3]. */
double nzo_lbc_viscosity(const nz_fluid_desc *f, const double *x, double rho, double T)
{
    const double psi = 0.45359237 * 9.80665 / (0.0254 * 0.0254);
    const double cp = 1.0e-3;
    const double kr = 5.0 / 9.0;
    double num = 0.0, den = 0.0, pc = 0.0, tc = 0.0, vc = 0.0, mw = 0.0;
    for (int i = 0; i < f->nc; ++i)
    {
        const double ms = sqrt(1000.0 * f->mw[i]);
        const double eps = 5.4402 * pow(f->tc[i] / kr, 1.0 / 6.0) / (ms * pow(f->pc[i] / psi, 2.0 / 3.0) * cp);
        const double tr = T / f->tc[i];
        const double mu = tr > 1.5 ? 17.78e-5 * pow(4.58 * tr - 1.67, 0.625) / eps
                                   : 34.0e-5 * pow(tr, 0.94) / eps;
        num += x[i] * mu * ms;
        den += x[i] * ms;
        pc += f->pc[i] * x[i];
        tc += f->tc[i] * x[i];
        vc += f->vc[i] * x[i];
        mw += f->mw[i] * x[i];
    }
    const double eps = 5.4402 * pow(tc / kr, 1.0 / 6.0) / (sqrt(1000.0 * mw) * pow(pc / psi, 2.0 / 3.0) * cp);
    const double r = vc * rho;
    const double p = 0.1023 + 0.023364 * r + 0.058533 * r * r - 0.040758 * r * r * r + 0.0093324 * r * r * r * r;
    return num / den + (p * p * p * p - 1.0e-4) / eps;
}
