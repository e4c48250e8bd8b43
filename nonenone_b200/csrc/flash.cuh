// flash.cuh -- device three-phase P-T-z flash, one thread per point, FP64.
//
// Restates the reference's CubicThreePhaseFlash
// (models/include/natural/thermo/three_phase_flash.hpp and
//  thermo/detail/three_phase_flash_{core,nonlinear,restricted,allocation,
//  canonicalization,stability}.inc) decision for decision: the same
// iteration caps, tolerances, finite-difference Newton steps, line searches,
// seed lists, canonicalisation passes and fail-only recovery order.  Line
// references below are to those files.
//
// Differences by design:
//  * exceptions become an error code in `err`; the flash then returns with
//    that status (the reference aborts the call with the exception);
//  * the SSI steps of the TPD trial reuse the fugacity coefficients of the
//    residual evaluation at the same composition (the reference evaluates
//    the EOS twice there; the EOS is deterministic so the values are equal);
//  * a restricted flash asked for all three phases (never requested by the
//    entry points carried here) returns NZ_FLASH_NOT_PORTED.
#pragma once

#include "eos.cuh"
#include "cpa.cuh"

namespace nz
{

template <int NC>
struct Result
{
    bool converged;
    int iterations;
    uint8_t presence;
    double beta[3];
    double sat[3];
    double x[3][NC];
    double Z[3];
    double rho[3];
    double Kg[NC];
    double Kw[NC];

    NZ_HDN void init()
    {
        converged = false;
        iterations = 0;
        presence = ALL_BITS;
        beta[0] = 1.0; beta[1] = 0.0; beta[2] = 0.0;
        sat[0] = 1.0; sat[1] = 0.0; sat[2] = 0.0;
        Z[0] = 1.0; Z[1] = 1.0; Z[2] = 1.0;
        rho[0] = 0.0; rho[1] = 0.0; rho[2] = 0.0;
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int i = 0; i < NC; ++i)
                x[p][i] = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            Kg[i] = 0.0;
            Kw[i] = 0.0;
        }
    }
};

#ifdef __CUDA_ARCH__
// `out` on every lane of the warp = `r` of lane `src` (all lanes call it).
template <int NC>
__device__ void shuffleResult(const Result<NC> &r, int src, Result<NC> &out)
{
    out.converged = __shfl_sync(0xffffffffu, int(r.converged), src) != 0;
    out.iterations = __shfl_sync(0xffffffffu, r.iterations, src);
    out.presence = uint8_t(__shfl_sync(0xffffffffu, int(r.presence), src));
    for (int p = 0; p < 3; ++p)
    {
        out.beta[p] = __shfl_sync(0xffffffffu, r.beta[p], src);
        out.sat[p] = __shfl_sync(0xffffffffu, r.sat[p], src);
        out.Z[p] = __shfl_sync(0xffffffffu, r.Z[p], src);
        out.rho[p] = __shfl_sync(0xffffffffu, r.rho[p], src);
        for (int i = 0; i < NC; ++i)
            out.x[p][i] = __shfl_sync(0xffffffffu, r.x[p][i], src);
    }
    for (int i = 0; i < NC; ++i)
    {
        out.Kg[i] = __shfl_sync(0xffffffffu, r.Kg[i], src);
        out.Kw[i] = __shfl_sync(0xffffffffu, r.Kw[i], src);
    }
}
#endif

// Outcome of one pressure-continuation anchor.
constexpr int CONT_NONE = 0;
constexpr int CONT_SUCCESS = 1;
constexpr int CONT_ERROR = 2;

template <int NC>
struct StabilityResult
{
    bool stable;
    bool valid;
    uint8_t tested;
    bool unstable[3];
    double incipient[3][NC];
    double trialSum[3];
};

template <int NC>
struct Trial
{
    bool valid;
    bool trivial;
    double sum;
    double x[NC];
};

template <int NC>
struct StabilityResidual
{
    bool valid;
    double norm;
    double sum;
    double x[NC];
    double residual[NC];
    double phi[NC];
    double lnphi[NC];   // set by the mixed-precision evaluation only
};

template <int NC>
struct TwoPhaseLogKState
{
    bool valid;
    double norm;
    double residual[NC];
    Result<NC> result;
};

template <int NC>
struct ThreePhaseLogKState
{
    bool valid;
    double norm;
    double residual[2 * NC];
    Result<NC> result;
};

// ---- small helpers ---------------------------------------------------------
NZ_HDI int firstActive(uint8_t b)
{
    return (b & OIL_BIT) ? OIL : ((b & GAS_BIT) ? GAS : WATER);
}

NZ_HDI void activePair(uint8_t b, int &first, int &second)
{
    int n = 0;
    first = OIL;
    second = GAS;
    for (int p = 0; p < 3; ++p)
    {
        if (b & bitOf(p))
        {
            if (n == 0) first = p;
            else if (n == 1) second = p;
            ++n;
        }
    }
}

// Dense Gaussian elimination with partial pivoting (stability.inc:98-146).
template <int M>
NZ_HD bool solveDense(double (&m)[M][M], double (&rhs)[M], double (&sol)[M])
{
#pragma unroll 1
    for (int k = 0; k < M; ++k)
        sol[k] = 0.0;
#pragma unroll 1
    for (int col = 0; col < M; ++col)
    {
        int pivot = col;
#pragma unroll 1
        for (int row = col + 1; row < M; ++row)
            if (fabs(m[row][col]) > fabs(m[pivot][col]))
                pivot = row;
        if (!(fabs(m[pivot][col]) > 1.0e-13))
            return false;
        if (pivot != col)
        {
#pragma unroll 1
            for (int j = 0; j < M; ++j)
            {
                const double t = m[pivot][j];
                m[pivot][j] = m[col][j];
                m[col][j] = t;
            }
            const double t = rhs[pivot];
            rhs[pivot] = rhs[col];
            rhs[col] = t;
        }
#pragma unroll 1
        for (int row = col + 1; row < M; ++row)
        {
            const double factor = m[row][col] / m[col][col];
            if (!isfinite(factor))
                return false;
#pragma unroll 1
            for (int j = col; j < M; ++j)
                m[row][j] -= factor * m[col][j];
            rhs[row] -= factor * rhs[col];
        }
    }
#pragma unroll 1
    for (int rev = 0; rev < M; ++rev)
    {
        const int row = M - 1 - rev;
        double value = rhs[row];
#pragma unroll 1
        for (int j = row + 1; j < M; ++j)
            value -= m[row][j] * sol[j];
        if (!(fabs(m[row][row]) > 1.0e-13))
            return false;
        sol[row] = value / m[row][row];
        if (!isfinite(sol[row]))
            return false;
    }
    return true;
}

// The SW role permutations (core.inc:37-45).
NZ_HDI void swRolePermutation(int k, int (&roles)[3])
{
    const int table[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    roles[0] = table[k][0];
    roles[1] = table[k][1];
    roles[2] = table[k][2];
}

// A robust three-phase Rachford-Rice answer computed ahead of time for one
// exact input (z, K_g, K_w and the preferred fractions).  rr3Robust returns it
// when it is called with bit-identical inputs and solves as usual otherwise.
template <int NC>
struct Rr3Memo
{
    double z[NC], kg[NC], kw[NC];
    double pg, pw;
    double bg, bw;
    int ok;
    int valid;

    NZ_HD bool matches(const double *zz, const double *g, const double *w, double ppg, double ppw) const
    {
        if (!valid || pg != ppg || pw != ppw)
            return false;
        for (int i = 0; i < NC; ++i)
            if (z[i] != zz[i] || kg[i] != g[i] || kw[i] != w[i])
                return false;
        return true;
    }
};

// A stability test computed ahead of time for one exact input (P, T, z, the
// active set and its compositions).  stabilityTest returns the stored answer
// when it is called with identical inputs and tests as usual otherwise.  The
// batched Natural update uses it to run the main-path test of every cell on
// the lane-per-trial kernel before the per-cell code runs.
constexpr uint8_t MEMO_NONE = 0;        // no test recorded
constexpr uint8_t MEMO_CAPTURED = 1;    // input recorded, answer pending
constexpr uint8_t MEMO_READY = 2;       // answer stored

template <int NC>
struct StabilityMemo
{
    double P, T;
    double z[NC];
    double x[3][NC];
    StabilityResult<NC> res;
    int err;
    uint8_t active;
    uint8_t state;

    NZ_HD void record(double p, double t, const double *zz, uint8_t act, const double (&xx)[3][NC])
    {
        P = p;
        T = t;
        active = act;
        for (int i = 0; i < NC; ++i)
            z[i] = zz[i];
        for (int q = 0; q < 3; ++q)
            for (int i = 0; i < NC; ++i)
                x[q][i] = xx[q][i];
        state = MEMO_CAPTURED;
    }

    NZ_HD bool matches(double p, double t, const double *zz, uint8_t act, const double (&xx)[3][NC]) const
    {
        if (state != MEMO_READY || P != p || T != t || active != act)
            return false;
        for (int i = 0; i < NC; ++i)
            if (z[i] != zz[i])
                return false;
        for (int q = 0; q < 3; ++q)
            for (int i = 0; i < NC; ++i)
                if (x[q][i] != xx[q][i])
                    return false;
        return true;
    }
};

// A top-level flash computed ahead of time (by the staged batched flash) for
// one exact input (P, T, z).  flash<true> returns it when called with
// identical inputs; `err` carries the flash's error code (0 = none).
template <int NC>
struct FlashMemo
{
    double P, T;
    double z[NC];
    Result<NC> r;
    int err;
    int valid;

    NZ_HD bool matches(double p, double t, const double *zz) const
    {
        if (!valid || P != p || T != t)
            return false;
        for (int i = 0; i < NC; ++i)
            if (z[i] != zz[i])
                return false;
        return true;
    }
};

// What one seed of the SW allocation search ends in (computed ahead of time
// by the staged batched flash, one lane per seed): admissible or not, the
// error it raised, its Gibbs energy and the three-phase allocation.
template <int NC>
struct AllocSeedOut
{
    double gibbs;
    double beta[3];
    double Z[3];
    double x[3][NC];
    int admissible;
    int err;
};

constexpr int kAllocSeedCount = 23;   // seeds of flashThreeAllocationFallback_ (allocation.inc:609-700)

// The allocation search of one exact input (P, T, salinity, z): every seed's
// outcome.  allocationFallback replays the sequential acceptance over them
// when it is called with identical inputs and the default phase roles.
template <int NC>
struct AllocMemo
{
    double P, T, salinity;
    double z[NC];
    int valid;
    AllocSeedOut<NC> seed[kAllocSeedCount];

    NZ_HD bool matches(double p, double t, double s, const double *zz) const
    {
        if (!valid || P != p || T != t || salinity != s)
            return false;
        for (int i = 0; i < NC; ++i)
            if (z[i] != zz[i])
                return false;
        return true;
    }
};

// The SW role-permutation search (three_phase_flash.hpp:174-205) of one exact
// input computed ahead of time: for each fixed role permutation k, the
// nested flash's answer, whether it is usable, its Gibbs energy under those
// roles and its error.  recover() replays the sequential choice over them.
template <int NC>
struct PermOut
{
    Result<NC> r;
    double gibbs;
    int ok;
    int err;
};

template <int NC>
struct PermMemo
{
    double P, T, salinity;
    double z[NC];
    int valid;
    PermOut<NC> perm[6];

    NZ_HD bool matches(double p, double t, double s, const double *zz) const
    {
        if (!valid || P != p || T != t || salinity != s)
            return false;
        for (int i = 0; i < NC; ++i)
            if (z[i] != zz[i])
                return false;
        return true;
    }
};

// ============================================================================
template <int NC>
struct Solver
{
    const FluidDev *F;
    double salinity;
    int roles[3];
    bool permutationSearch;
    bool continuation;
    int err;
    unsigned long long evals;
    // Warp-cooperative mode: all `width` lanes run the same point in lockstep
    // and split the seeds of every stability test (width 1 = one thread).
    int lane;
    int width;
    // cubic parameter cache (core.inc:71-99)
    bool cacheValid;
    double cacheP, cacheT;
    MixParams<NC> nonAq;
    MixParams<NC> aq;
    const Rr3Memo<NC> *memo;   // optional precomputed rr3Robust answer
    StabilityMemo<NC> *stabMemo;   // optional precomputed stability test
    const FlashMemo<NC> *flashMemo;   // optional precomputed top-level flash
    const AllocMemo<NC> *allocMemo;   // optional precomputed SW allocation seeds
    const PermMemo<NC> *permMemo;     // optional precomputed SW role-permutation search
    // Staged use: stop recover() where the role-permutation search would
    // start (reachedPermutations tells), so that it can be run ahead.
    bool stopAtPermutations;
    bool reachedPermutations;
    bool mixed;                    // mixed-precision successive substitution in the TPD trials

    NZ_HD void setup(const FluidDev *fluid, double s)
    {
        F = fluid;
        salinity = s;
        roles[0] = OIL; roles[1] = GAS; roles[2] = WATER;
        permutationSearch = true;
        continuation = true;
        err = ERR_NONE;
        evals = 0;
        lane = 0;
        width = 1;
        cacheValid = false;
        cacheP = cacheT = 0.0;
        memo = nullptr;
        stabMemo = nullptr;
        flashMemo = nullptr;
        allocMemo = nullptr;
        permMemo = nullptr;
        stopAtPermutations = false;
        reachedPermutations = false;
        mixed = false;
    }

    NZ_HD const FlashOpts &O() const { return F->opt; }
    NZ_HD bool sw() const { return F->eosModel == EOS_SW; }

    NZ_HD void fail(int code)
    {
        if (err == ERR_NONE)
            err = code;
    }

    // ---------------------------------------------------------------- core --
    NZ_HD int thermodynamicRole(int slot) const { return sw() ? roles[slot] : slot; }

    NZ_HD void ensureCache(double P, double T)
    {
        if (cacheValid && cacheP == P && cacheT == T)
            return;
        mixingParameters<NC>(*F, P, T, salinity, false, nonAq);
        if (sw())
            mixingParameters<NC>(*F, P, T, salinity, true, aq);
        cacheP = P;
        cacheT = T;
        cacheValid = true;
    }

    // phaseResultForThermodynamicRole_ (core.inc:101-126)
    NZ_HDN double phaseForRole(int role, double P, double T, const double *x, double *phi)
    {
        if (F->eosModel == EOS_CPA)
        {
            // phaseResult's CPA branch (core.inc:108-112 -> cubic_eos.hpp:842-846)
            ++evals;
            double Z = 0.0;
            const int rc = cpaPhase<NC>(*F, P, T, x, role != GAS, Z, phi);
            if (rc != ERR_NONE)
            {
                fail(rc);
                const double nan = nzNan();
                for (int i = 0; i < NC; ++i)
                    phi[i] = nan;
                return nan;
            }
            return Z;
        }
        ensureCache(P, T);
        const MixParams<NC> &p = (role == WATER && sw()) ? aq : nonAq;
        PhaseMix<NC> m;
        phaseMixing<NC>(x, p, m);
        ++evals;
        const double Z = selectCubicRoot(m.A, m.B, F->m1, F->m2, role == GAS);
        if (!isfinite(Z) || !fugacityCoefficients<NC>(x, p, m, Z, F->m1, F->m2, phi))
        {
            fail(ERR_EOS);
            const double nan = nzNan();
#pragma unroll
            for (int i = 0; i < NC; ++i)
                phi[i] = nan;
            return nan;
        }
        return Z;
    }

    NZ_HD double phase(int slot, double P, double T, const double *x, double *phi)
    {
        return phaseForRole(thermodynamicRole(slot), P, T, x, phi);
    }

    NZ_HD bool validatePT(double P, double T)
    {
        if (!(P > 0.0) || !isfinite(P) || !(T > 0.0) || !isfinite(T))
        {
            fail(ERR_BAD_INPUT);
            return false;
        }
        return true;
    }

    // normalize_ (core.inc:136-149)
    NZ_HD void normalize(double *x)
    {
        double sum = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            if (!isfinite(x[i]))
                fail(ERR_BAD_INPUT);
            x[i] = smax(x[i], O().floor);
            sum += x[i];
        }
        if (!(sum > 0.0))
            fail(ERR_BAD_INPUT);
#pragma unroll
        for (int i = 0; i < NC; ++i)
            x[i] /= sum;
    }

    // wilsonGasOilK_ (core.inc:152-165)
    NZ_HD void wilsonK(double P, double T, double *K) const
    {
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double lnK = log(F->pc[i] / P) + 5.373 * (1.0 + F->omega[i]) * (1.0 - F->tc[i] / T);
            K[i] = sclamp(exp(lnK), 1.0e-30, 1.0e30);
        }
    }

    // initialWaterOilK_ (core.inc:168-176)
    NZ_HD void initialWaterK(double *K) const
    {
#pragma unroll
        for (int i = 0; i < NC; ++i)
            K[i] = 0.05;
        K[F->water >= 0 ? F->water : NC - 1] = 50.0;
    }

    NZ_HD uint8_t presenceFromFractions(const double *beta) const
    {
        uint8_t b = 0;
        for (int p = 0; p < 3; ++p)
            if (beta[p] > O().betaTol)
                b |= uint8_t(bitOf(p));
        return b;
    }

    // ------------------------------------------------------- Rachford-Rice --
    // residual/Jacobian of the three-phase RR (nonlinear.inc:30-58)
    NZ_HD double rr3Norm(const double *z, const double *kg, const double *kw, double cg, double cw,
                              double &fg, double &fw, double &jgg, double &jww, double &jgw) const
    {
        const double inf = nzInf();
        if (!(cg > 0.0) || !(cw > 0.0) || !(cg + cw < 1.0))
            return inf;
        fg = 0.0; fw = 0.0; jgg = 0.0; jww = 0.0; jgw = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double ag = kg[i] - 1.0;
            const double aw = kw[i] - 1.0;
            const double co = 1.0 - cg - cw;
            const double D = co + cg * kg[i] + cw * kw[i];
            if (!(D > 1.0e-12) || !isfinite(D))
                return inf;
            fg += z[i] * ag / D;
            fw += z[i] * aw / D;
            const double invD2 = z[i] / (D * D);
            jgg -= invD2 * ag * ag;
            jww -= invD2 * aw * aw;
            jgw -= invD2 * ag * aw;
        }
        return smax(fabs(fg), fabs(fw));
    }

    // solveRr3_ (nonlinear.inc:8-96)
    NZ_HDN bool rr3(const double *z, const double *kg, const double *kw, double initBg, double initBw,
                        double &outBg, double &outBw) const
    {
        double bg = sclamp(initBg, 1.0e-4, 0.8);
        double bw = sclamp(initBw, 1.0e-4, 0.8);
        if (bg + bw >= 0.95)
        {
            const double scale = 0.8 / (bg + bw);
            bg *= scale;
            bw *= scale;
        }
#pragma unroll 1
        for (int it = 0; it < O().maxRr; ++it)
        {
            double fg, fw, jgg, jww, jgw;
            const double norm = rr3Norm(z, kg, kw, bg, bw, fg, fw, jgg, jww, jgw);
            if (!isfinite(norm))
                return false;
            if (norm < O().rrTol)
            {
                outBg = bg;
                outBw = bw;
                return true;
            }
            const double det = jgg * jww - jgw * jgw;
            if (fabs(det) < 1.0e-24 || !isfinite(det))
                return false;
            const double dbg = (-fg * jww + fw * jgw) / det;
            const double dbw = (-fw * jgg + fg * jgw) / det;
            double lambda = 1.0;
            bool accepted = false;
#pragma unroll 1
            for (int ls = 0; ls < 40; ++ls)
            {
                const double cg = bg + lambda * dbg;
                const double cw = bw + lambda * dbw;
                double a, b, c, d, e;
                const double cn = rr3Norm(z, kg, kw, cg, cw, a, b, c, d, e);
                if (isfinite(cn) && cn < norm)
                {
                    bg = cg;
                    bw = cw;
                    accepted = true;
                    break;
                }
                lambda *= 0.5;
            }
            if (!accepted)
                return false;
        }
        return false;
    }

    // solveRr3Robust_ (nonlinear.inc:98-127)
    NZ_HDN bool rr3Robust(const double *z, const double *kg, const double *kw, double pg, double pw,
                              double &bg, double &bw) const
    {
        const double guesses[17][2] = {
            {pg, pw}, {0.333, 0.333}, {0.50, 1.0e-4}, {1.0e-4, 0.50}, {0.80, 1.0e-4},
            {1.0e-4, 0.80}, {0.20, 0.20}, {0.60, 0.20}, {0.20, 0.60}, {0.05, 0.05},
            {0.90, 0.01}, {0.95, 1.0e-4}, {0.98, 1.0e-4}, {1.0e-4, 0.95}, {1.0e-4, 0.98},
            {0.01, 0.90}, {0.45, 0.45}};
        if (memo && memo->matches(z, kg, kw, pg, pw))
        {
            if (!memo->ok)
                return false;
            bg = memo->bg;
            bw = memo->bw;
            return true;
        }
#ifdef __CUDA_ARCH__
        if (width > 1)
        {
            // Warp-cooperative: the preferred start on every lane (it usually
            // converges), then the other 16 starts spread over the lanes.  Each
            // start is an independent deterministic solve, so taking the lowest
            // converged start reproduces the sequential first-success rule.
            if (rr3(z, kg, kw, guesses[0][0], guesses[0][1], bg, bw))
                return true;
            int found = 0x7fffffff;
            double lg = 0.0, lw = 0.0;
#pragma unroll 1
            for (int g = 1 + lane; g < 17; g += width)
                if (rr3(z, kg, kw, guesses[g][0], guesses[g][1], lg, lw))
                {
                    found = g;
                    break;
                }
            __syncwarp();
            int first = found;
            for (int off = 16; off > 0; off >>= 1)
                first = imin(first, __shfl_xor_sync(0xffffffffu, first, off));
            if (first == 0x7fffffff)
                return false;
            const int src = (first - 1) % width;
            bg = __shfl_sync(0xffffffffu, lg, src);
            bw = __shfl_sync(0xffffffffu, lw, src);
            return true;
        }
#endif
#pragma unroll 1
        for (int g = 0; g < 17; ++g)
            if (rr3(z, kg, kw, guesses[g][0], guesses[g][1], bg, bw))
                return true;
        return false;
    }

    // solveRr2_ (nonlinear.inc:129-187)
    NZ_HD double rr2Eval(const double *z, const double *K, double beta, double &df) const
    {
        double f = 0.0;
        df = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double a = K[i] - 1.0;
            const double D = (1.0 - beta) + beta * K[i];
            if (!(D > 1.0e-300) || !isfinite(D))
                return nzNan();
            f += z[i] * a / D;
            df -= z[i] * a * a / (D * D);
        }
        return f;
    }

    NZ_HDN bool rr2(const double *z, const double *K, double initialBeta, double &out) const
    {
        double d0;
        const double f0 = rr2Eval(z, K, 0.0, d0);
        const double f1 = rr2Eval(z, K, 1.0, d0);
        if (!isfinite(f0) || !isfinite(f1))
            return false;
        if (f0 <= 0.0)
        {
            out = 0.0;
            return true;
        }
        if (f1 >= 0.0)
        {
            out = 1.0;
            return true;
        }
        double lower = 0.0, upper = 1.0;
        double beta = sclamp(initialBeta, lower, upper);
#pragma unroll 1
        for (int it = 0; it < O().maxRr; ++it)
        {
            double df;
            const double f = rr2Eval(z, K, beta, df);
            if (!isfinite(f) || !isfinite(df))
                return false;
            if (fabs(f) < O().rrTol)
            {
                out = beta;
                return true;
            }
            if (f > 0.0) lower = beta; else upper = beta;
            double candidate = beta;
            if (fabs(df) > 1.0e-24)
                candidate = beta - f / df;
            if (!isfinite(candidate) || candidate <= lower || candidate >= upper)
                candidate = 0.5 * (lower + upper);
            beta = candidate;
        }
        return false;
    }

    // ----------------------------------------------------- result helpers --
    // deriveReferenceK_ (restricted.inc:414-423)
    NZ_HD void deriveReferenceK(Result<NC> &r) const
    {
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double xo = smax(r.x[0][i], O().floor);
            r.Kg[i] = r.x[1][i] / xo;
            r.Kw[i] = r.x[2][i] / xo;
        }
    }

    // updateSaturationsFromMoles (three_phase_flash.hpp:527-575).  No aqueous
    // volume closure is configured, so every Water composition is admissible.
    NZ_HDN void updateSaturations(double P, double T, Result<NC> &r)
    {
        double volumeSum = 0.0;
        double volume[3] = {0.0, 0.0, 0.0};
        for (int p = 0; p < 3; ++p)
        {
            if (!(r.presence & bitOf(p)))
            {
                r.beta[p] = 0.0;
                r.sat[p] = 0.0;
                r.rho[p] = 0.0;
                continue;
            }
            const double Z = r.Z[p];
            if (!(Z > 0.0))
            {
                fail(ERR_EOS);
                return;
            }
            const double rhoM = molarDensity(P, T, Z);
            r.rho[p] = rhoM;
            volume[p] = smax(r.beta[p], 0.0) / rhoM;
            volumeSum += volume[p];
        }
        if (!(volumeSum > 0.0))
        {
            fail(ERR_EOS);
            return;
        }
        for (int p = 0; p < 3; ++p)
            r.sat[p] = volume[p] / volumeSum;
    }

    // singlePhaseResult_ (restricted.inc:425-447)
    NZ_HDN void singlePhaseResult(double P, double T, const double *z, uint8_t active, Result<NC> &r)
    {
        r.init();
        r.converged = true;
        r.presence = active;
        r.beta[0] = r.beta[1] = r.beta[2] = 0.0;
        const int p = firstActive(active);
        r.beta[p] = 1.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
            r.x[p][i] = z[i];
        for (int q = 0; q < 3; ++q)
            if (!(active & bitOf(q)))
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    r.x[q][i] = z[i];
        double phi[NC];
        r.Z[p] = phase(p, P, T, z, phi);
        deriveReferenceK(r);
        updateSaturations(P, T, r);
    }

    // waterIsDominant_ (canonicalization.inc:68-85)
    NZ_HD bool waterIsDominant(const double *x) const
    {
        if (F->water < 0)
            return false;
        double largestOther = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
            if (i != F->water)
                largestOther = smax(largestOther, x[i]);
        return x[F->water] >= largestOther;
    }

    // chooseSinglePhase_ (restricted.inc:449-478)
    NZ_HDN uint8_t chooseSinglePhase(double P, double T, const double *z)
    {
        double phi[NC];
        double g[3];
        for (int p = 0; p < 3; ++p)
        {
            phase(p, P, T, z, phi);
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                s += z[i] * log(smax(phi[i], 1.0e-300));
            g[p] = s;
        }
        const double go = g[0], gg = g[1], gw = g[2];
        const double tie = 1.0e-10;
        if (gg + tie < go && gg + tie < gw)
            return GAS_BIT;
        if (gw + tie < go && gw + tie < gg)
            return WATER_BIT;
        if (waterIsDominant(z) && fabs(gw - go) <= tie)
            return WATER_BIT;
        if (gg + tie < go)
            return GAS_BIT;
        return OIL_BIT;
    }

    // dimensionlessGibbs_ (restricted.inc:480-505); the public slot is the role.
    NZ_HDN double dimensionlessGibbs(double P, double T, const Result<NC> &r)
    {
        double g = 0.0;
        double phi[NC];
        for (int p = 0; p < 3; ++p)
        {
            const double beta = r.beta[p];
            if (!(beta > O().betaTol))
                continue;
            phaseForRole(p, P, T, r.x[p], phi);
#pragma unroll
            for (int i = 0; i < NC; ++i)
            {
                const double xi = smax(r.x[p][i], O().floor);
                const double ph = smax(phi[i], 1.0e-300);
                g += beta * r.x[p][i] * (log(xi) + log(ph));
            }
        }
        return g;
    }

    NZ_HD void swapSlots(Result<NC> &r, int a, int b) const
    {
        if (a == b)
            return;
        double t;
        t = r.beta[a]; r.beta[a] = r.beta[b]; r.beta[b] = t;
        t = r.sat[a]; r.sat[a] = r.sat[b]; r.sat[b] = t;
        t = r.Z[a]; r.Z[a] = r.Z[b]; r.Z[b] = t;
        t = r.rho[a]; r.rho[a] = r.rho[b]; r.rho[b] = t;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            t = r.x[a][i]; r.x[a][i] = r.x[b][i]; r.x[b][i] = t;
        }
    }

    // ------------------------------------------------------- pair seeds ----
    // pairInitialK_ (nonlinear.inc:515-623)
    NZ_HDN void pairInitialK(int first, int second, double P, double T, const double *z, double *K)
    {
        if (sw() && (first == WATER || second == WATER))
        {
            const int water = F->water >= 0 ? F->water : NC - 1;
            double seeds[2][NC];
            const int which[2] = {first, second};
            for (int s = 0; s < 2; ++s)
            {
                double *seed = seeds[s];
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    seed[i] = z[i];
                if (which[s] == WATER)
                {
                    double nonWater = 0.0;
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                    {
                        if (i == water) continue;
                        seed[i] = smax(z[i], O().floor);
                        nonWater += seed[i];
                    }
                    const double dissolved = 0.02;
                    if (nonWater > 0.0)
#pragma unroll
                        for (int i = 0; i < NC; ++i)
                            if (i != water)
                                seed[i] *= dissolved / nonWater;
                    seed[water] = 1.0 - dissolved;
                }
                else
                {
                    const double waterSeed = 0.01;
                    double nonWater = 0.0;
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                        if (i != water)
                            nonWater += smax(z[i], O().floor);
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                    {
                        if (i == water)
                            seed[i] = waterSeed;
                        else
                            seed[i] = nonWater > 0.0
                                ? (1.0 - waterSeed) * smax(z[i], O().floor) / nonWater
                                : (1.0 - waterSeed) / double(NC - 1 > 1 ? NC - 1 : 1);
                    }
                }
                normalize(seed);
            }
            double phiA[NC], phiB[NC];
            phase(first, P, T, seeds[0], phiA);
            phase(second, P, T, seeds[1], phiB);
#pragma unroll
            for (int i = 0; i < NC; ++i)
                K[i] = sclamp(smax(phiA[i], 1.0e-300) / smax(phiB[i], 1.0e-300), 1.0e-100, 1.0e100);
            return;
        }
        double kg[NC], kw[NC];
        wilsonK(P, T, kg);
        initialWaterK(kw);
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double rs = second == OIL ? 1.0 : (second == GAS ? kg[i] : kw[i]);
            const double rf = first == OIL ? 1.0 : (first == GAS ? kg[i] : kw[i]);
            K[i] = rs / rf;
        }
    }

    // --------------------------------------------------------- two-phase ---
    // evaluateTwoPhaseLogK_ (restricted.inc:71-134)
    NZ_HDN void evalTwo(double P, double T, const double *z, int first, int second,
                                         const double *logK, double preferredSecond,
                                         TwoPhaseLogKState<NC> &s)
    {
        s.valid = false;
        s.norm = nzInf();
        s.result.init();
        double K[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            K[i] = exp(sclamp(logK[i], -230.0, 230.0));
        double bS;
        if (!rr2(z, K, preferredSecond, bS))
            return;
        const double bF = 1.0 - bS;
        double a[NC], b[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double D = (1.0 - bS) + bS * K[i];
            if (!(D > 0.0) || !isfinite(D))
                return;
            a[i] = z[i] / D;
            b[i] = K[i] * a[i];
        }
        normalize(a);
        normalize(b);
        double phiA[NC], phiB[NC];
        const double ZA = phase(first, P, T, a, phiA);
        const double ZB = phase(second, P, T, b, phiB);
        s.norm = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double pa = smax(phiA[i], 1.0e-300);
            const double pb = smax(phiB[i], 1.0e-300);
            s.residual[i] = logK[i] - log(pa / pb);
            s.norm = smax(s.norm, fabs(s.residual[i]));
        }
        Result<NC> &r = s.result;
        r.presence = uint8_t(bitOf(first) | bitOf(second));
        r.beta[0] = r.beta[1] = r.beta[2] = 0.0;
        r.beta[first] = bF;
        r.beta[second] = bS;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            r.x[first][i] = a[i];
            r.x[second][i] = b[i];
        }
        r.Z[first] = ZA;
        r.Z[second] = ZB;
        for (int p = 0; p < 3; ++p)
            if (!(r.presence & bitOf(p)))
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    r.x[p][i] = z[i];
        s.valid = isfinite(s.norm);
    }

    // one damped SSI step of flashTwo_ (restricted.inc:155-208)
    NZ_HDN bool twoSsiStep(double P, double T, const double *z, int first, int second, double *K,
                               double &betaSecond, int &totalIterations, Result<NC> &r)
    {
        double bS;
        if (!rr2(z, K, betaSecond, bS))
            return false;
        betaSecond = bS;
        const double bF = 1.0 - bS;
        double a[NC], b[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double D = (1.0 - bS) + bS * K[i];
            if (!(D > 0.0) || !isfinite(D))
                return false;
            a[i] = z[i] / D;
            b[i] = K[i] * a[i];
        }
        normalize(a);
        normalize(b);
        double phiA[NC], phiB[NC];
        const double ZA = phase(first, P, T, a, phiA);
        const double ZB = phase(second, P, T, b, phiB);
        double maxResidual = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double target = smax(phiA[i], 1.0e-300) / smax(phiB[i], 1.0e-300);
            const double d = sclamp(log(target / K[i]), -O().logKLimit, O().logKLimit);
            maxResidual = smax(maxResidual, fabs(d));
            K[i] *= exp(0.6 * d);
            K[i] = sclamp(K[i], 1.0e-100, 1.0e100);
        }
        ++totalIterations;
        r.iterations = totalIterations;
        r.beta[0] = r.beta[1] = r.beta[2] = 0.0;
        r.beta[first] = bF;
        r.beta[second] = bS;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            r.x[first][i] = a[i];
            r.x[second][i] = b[i];
        }
        r.Z[first] = ZA;
        r.Z[second] = ZB;
        for (int p = 0; p < 3; ++p)
            if (!(r.presence & bitOf(p)))
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    r.x[p][i] = z[i];
        if (maxResidual < O().fugacityTol)
        {
            r.converged = true;
            r.presence = presenceFromFractions(r.beta);
            deriveReferenceK(r);
            updateSaturations(P, T, r);
        }
        return true;
    }

    // flashTwo_ (restricted.inc:136-327)
    NZ_HDN void flashTwo(double P, double T, const double *z, int first, int second,
                                          const double *Kin, Result<NC> &r)
    {
        r.init();
        r.presence = uint8_t(bitOf(first) | bitOf(second));
        double K[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            K[i] = sclamp(Kin[i], 1.0e-100, 1.0e100);
        double betaSecond = 0.5;
        int total = 0;
        const int ssiSteps = imin(O().maxIterations, imax(O().twoSsi, 0));
#pragma unroll 1
        for (int it = 0; it < ssiSteps; ++it)
        {
            if (!twoSsiStep(P, T, z, first, second, K, betaSecond, total, r))
                return;
            if (r.converged || err)
                return;
        }
        double logK[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            logK[i] = log(K[i]);

        TwoPhaseLogKState<NC> base, probe;
#pragma unroll 1
        for (int it = 0; it < O().twoNewton; ++it)
        {
            evalTwo(P, T, z, first, second, logK, betaSecond, base);
            if (!base.valid || err)
                break;
            r = base.result;
            r.iterations = ++total;
            betaSecond = r.beta[second];
            if (base.norm < O().fugacityTol)
            {
                r.converged = true;
                r.presence = presenceFromFractions(r.beta);
                deriveReferenceK(r);
                updateSaturations(P, T, r);
                return;
            }
            double J[NC][NC];
            bool jacobianValid = true;
#pragma unroll 1
            for (int col = 0; col < NC; ++col)
            {
                double pert[NC];
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    pert[i] = logK[i];
                const double step = O().fdStep * smax(1.0, fabs(logK[col]));
                pert[col] += step;
                evalTwo(P, T, z, first, second, pert, betaSecond, probe);
                if (!probe.valid)
                {
                    jacobianValid = false;
                    break;
                }
#pragma unroll
                for (int row = 0; row < NC; ++row)
                    J[row][col] = (probe.residual[row] - base.residual[row]) / step;
            }
            if (!jacobianValid)
                break;
            double rhs[NC], delta[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i)
                rhs[i] = -base.residual[i];
            if (!solveDense<NC>(J, rhs, delta))
                break;
            bool accepted = false;
            double damping = 1.0;
#pragma unroll 1
            for (int ls = 0; ls < 16; ++ls)
            {
                double trialLogK[NC];
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    trialLogK[i] = logK[i] + damping * delta[i];
                evalTwo(P, T, z, first, second, trialLogK, betaSecond, probe);
                if (probe.valid && probe.norm < base.norm)
                {
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                        logK[i] = trialLogK[i];
                    accepted = true;
                    break;
                }
                damping *= 0.5;
            }
            if (!accepted)
                break;
        }
#pragma unroll 1
        for (int it = ssiSteps; it < O().maxIterations; ++it)
        {
            if (err)
                return;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                K[i] = exp(sclamp(logK[i], -230.0, 230.0));
            if (!twoSsiStep(P, T, z, first, second, K, betaSecond, total, r))
                return;
            if (r.converged)
                return;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                logK[i] = log(K[i]);
        }
    }

    // finalizePhysicallyConvergedTwoPhase_ (restricted.inc:336-412)
    NZ_HDN void finalizePhysicallyConvergedTwoPhase(double P, double T, const double *z, int first,
                                                        int second, Result<NC> &r)
    {
        if (r.converged)
            return;
        const double betaA = r.beta[first];
        const double betaB = r.beta[second];
        if (!(betaA > O().betaTol) || !(betaB > O().betaTol) || !isfinite(betaA) || !isfinite(betaB))
            return;
        const double betaClosure = fabs(betaA + betaB - 1.0);
        const double closureTol = smax(O().fugacityTol, 10.0 * O().rrTol);
        if (betaClosure > closureTol)
            return;
        double xa[NC], xb[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            xa[i] = r.x[first][i];
            xb[i] = r.x[second][i];
        }
        normalize(xa);
        normalize(xb);
        double materialClosure = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double rec = betaA * xa[i] + betaB * xb[i];
            materialClosure = smax(materialClosure, fabs(rec - z[i]));
        }
        if (materialClosure > closureTol)
            return;
        double phiA[NC], phiB[NC];
        const double ZA = phase(first, P, T, xa, phiA);
        const double ZB = phase(second, P, T, xb, phiB);
        double fugacityResidual = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double aA = smax(xa[i] * phiA[i], 1.0e-300);
            const double aB = smax(xb[i] * phiB[i], 1.0e-300);
            fugacityResidual = smax(fugacityResidual, fabs(log(aA / aB)));
        }
        if (fugacityResidual > O().fugacityTol)
            return;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            r.x[first][i] = xa[i];
            r.x[second][i] = xb[i];
        }
        r.presence = uint8_t(bitOf(first) | bitOf(second));
        r.Z[first] = ZA;
        r.Z[second] = ZB;
        r.converged = true;
        deriveReferenceK(r);
        updateSaturations(P, T, r);
    }

    // ------------------------------------------------------- three-phase ---
    // evaluateThreePhaseLogK_ (nonlinear.inc:200-277)
    NZ_HDN void evalThree(double P, double T, const double *z, const double *logK,
                                           double preferredGas, double preferredWater,
                                           ThreePhaseLogKState<NC> &s)
    {
        s.valid = false;
        s.norm = nzInf();
        s.result.init();
        double kg[NC], kw[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            kg[i] = exp(sclamp(logK[i], -230.0, 230.0));
            kw[i] = exp(sclamp(logK[NC + i], -230.0, 230.0));
        }
        double bg, bw;
        if (!rr3Robust(z, kg, kw, preferredGas, preferredWater, bg, bw))
            return;
        const double bo = 1.0 - bg - bw;
        if (!(bo >= -O().betaTol) || !(bg >= -O().betaTol) || !(bw >= -O().betaTol))
            return;
        double xo[NC], yg[NC], xw[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double D = bo + bg * kg[i] + bw * kw[i];
            if (!(D > 0.0) || !isfinite(D))
                return;
            xo[i] = z[i] / D;
            yg[i] = kg[i] * xo[i];
            xw[i] = kw[i] * xo[i];
        }
        normalize(xo);
        normalize(yg);
        normalize(xw);
        double phiO[NC], phiG[NC], phiW[NC];
        const double Zo = phase(OIL, P, T, xo, phiO);
        const double Zg = phase(GAS, P, T, yg, phiG);
        const double Zw = phase(WATER, P, T, xw, phiW);
        s.norm = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double po = smax(phiO[i], 1.0e-300);
            const double pg = smax(phiG[i], 1.0e-300);
            const double pw = smax(phiW[i], 1.0e-300);
            s.residual[i] = logK[i] - log(po / pg);
            s.residual[NC + i] = logK[NC + i] - log(po / pw);
            s.norm = smax3(s.norm, fabs(s.residual[i]), fabs(s.residual[NC + i]));
        }
        Result<NC> &r = s.result;
        r.presence = ALL_BITS;
        r.beta[0] = bo; r.beta[1] = bg; r.beta[2] = bw;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            r.x[0][i] = xo[i];
            r.x[1][i] = yg[i];
            r.x[2][i] = xw[i];
            r.Kg[i] = kg[i];
            r.Kw[i] = kw[i];
        }
        r.Z[0] = Zo; r.Z[1] = Zg; r.Z[2] = Zw;
        s.valid = isfinite(s.norm);
    }

    // one damped SSI step of flashThree_ (nonlinear.inc:301-371)
    NZ_HDN bool threeSsiStep(double P, double T, const double *z, double *kg, double *kw,
                                 double &bg, double &bw, int &total, Result<NC> &r)
    {
        double ng, nw;
        if (!rr3Robust(z, kg, kw, bg, bw, ng, nw))
            return false;
        bg = ng;
        bw = nw;
        const double bo = 1.0 - bg - bw;
        double xo[NC], yg[NC], xw[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double D = bo + bg * kg[i] + bw * kw[i];
            if (!(D > 0.0) || !isfinite(D))
                return false;
            xo[i] = z[i] / D;
            yg[i] = kg[i] * xo[i];
            xw[i] = kw[i] * xo[i];
        }
        normalize(xo);
        normalize(yg);
        normalize(xw);
        double phiO[NC], phiG[NC], phiW[NC];
        const double Zo = phase(OIL, P, T, xo, phiO);
        const double Zg = phase(GAS, P, T, yg, phiG);
        const double Zw = phase(WATER, P, T, xw, phiW);
        double maxResidual = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double po = smax(phiO[i], 1.0e-300);
            const double targetKg = po / smax(phiG[i], 1.0e-300);
            const double targetKw = po / smax(phiW[i], 1.0e-300);
            const double dg = sclamp(log(targetKg / kg[i]), -O().logKLimit, O().logKLimit);
            const double dw = sclamp(log(targetKw / kw[i]), -O().logKLimit, O().logKLimit);
            maxResidual = smax3(maxResidual, fabs(dg), fabs(dw));
            kg[i] *= exp(0.6 * dg);
            kw[i] *= exp(0.6 * dw);
            kg[i] = sclamp(kg[i], 1.0e-100, 1.0e100);
            kw[i] = sclamp(kw[i], 1.0e-100, 1.0e100);
        }
        ++total;
        r.iterations = total;
        r.beta[0] = bo; r.beta[1] = bg; r.beta[2] = bw;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            r.x[0][i] = xo[i];
            r.x[1][i] = yg[i];
            r.x[2][i] = xw[i];
            r.Kg[i] = kg[i];
            r.Kw[i] = kw[i];
        }
        r.Z[0] = Zo; r.Z[1] = Zg; r.Z[2] = Zw;
        if (maxResidual < O().fugacityTol)
        {
            r.converged = true;
            r.presence = presenceFromFractions(r.beta);
            updateSaturations(P, T, r);
        }
        return true;
    }

    // flashThree_ (nonlinear.inc:279-513)
    NZ_HDN void flashThree(double P, double T, const double *z, const double *kgIn,
                                            const double *kwIn, Result<NC> &r)
    {
        r.init();
        r.presence = ALL_BITS;
        double kg[NC], kw[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            kg[i] = sclamp(kgIn[i], 1.0e-100, 1.0e100);
            kw[i] = sclamp(kwIn[i], 1.0e-100, 1.0e100);
        }
        double bg = 0.15, bw = 0.15;
        const int ssiSteps = imin(O().maxIterations, imax(O().threeSsi, 0));
        int total = 0;
#pragma unroll 1
        for (int it = 0; it < ssiSteps; ++it)
        {
            if (!threeSsiStep(P, T, z, kg, kw, bg, bw, total, r))
                return;
            if (r.converged || err)
                return;
        }
        constexpr int M = 2 * NC;
        double logK[M];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            logK[i] = log(kg[i]);
            logK[NC + i] = log(kw[i]);
        }
        ThreePhaseLogKState<NC> base, probe;
#pragma unroll 1
        for (int it = 0; it < O().threeNewton; ++it)
        {
            evalThree(P, T, z, logK, bg, bw, base);
            if (!base.valid || err)
                break;
            r = base.result;
            r.iterations = ++total;
            bg = r.beta[1];
            bw = r.beta[2];
            if (base.norm < O().fugacityTol)
            {
                r.converged = true;
                r.presence = presenceFromFractions(r.beta);
                updateSaturations(P, T, r);
                return;
            }
            double J[M][M];
            bool jacobianValid = true;
#pragma unroll 1
            for (int col = 0; col < M; ++col)
            {
                const double step = O().fdStep * smax(1.0, fabs(logK[col]));
                double pert[M];
#pragma unroll
                for (int i = 0; i < M; ++i)
                    pert[i] = logK[i];
                pert[col] += step;
                evalThree(P, T, z, pert, bg, bw, probe);
                if (probe.valid)
                {
#pragma unroll
                    for (int row = 0; row < M; ++row)
                        J[row][col] = (probe.residual[row] - base.residual[row]) / step;
                    continue;
                }
#pragma unroll
                for (int i = 0; i < M; ++i)
                    pert[i] = logK[i];
                pert[col] -= step;
                evalThree(P, T, z, pert, bg, bw, probe);
                if (!probe.valid)
                {
                    jacobianValid = false;
                    break;
                }
#pragma unroll
                for (int row = 0; row < M; ++row)
                    J[row][col] = (base.residual[row] - probe.residual[row]) / step;
            }
            if (!jacobianValid)
                break;
            double rhs[M], delta[M];
#pragma unroll
            for (int i = 0; i < M; ++i)
                rhs[i] = -base.residual[i];
            if (!solveDense<M>(J, rhs, delta))
                break;
            bool accepted = false;
            double damping = 1.0;
#pragma unroll 1
            for (int ls = 0; ls < 16; ++ls)
            {
                double trialLogK[M];
#pragma unroll
                for (int i = 0; i < M; ++i)
                    trialLogK[i] = logK[i] + damping * delta[i];
                evalThree(P, T, z, trialLogK, bg, bw, probe);
                if (probe.valid && probe.norm < base.norm)
                {
#pragma unroll
                    for (int i = 0; i < M; ++i)
                        logK[i] = trialLogK[i];
                    accepted = true;
                    break;
                }
                damping *= 0.5;
            }
            if (!accepted)
                break;
        }
#pragma unroll 1
        for (int it = ssiSteps; it < O().maxIterations; ++it)
        {
            if (err)
                return;
#pragma unroll
            for (int i = 0; i < NC; ++i)
            {
                kg[i] = exp(sclamp(logK[i], -230.0, 230.0));
                kw[i] = exp(sclamp(logK[NC + i], -230.0, 230.0));
            }
            if (!threeSsiStep(P, T, z, kg, kw, bg, bw, total, r))
                return;
            if (r.converged)
                return;
#pragma unroll
            for (int i = 0; i < NC; ++i)
            {
                logK[i] = log(kg[i]);
                logK[NC + i] = log(kw[i]);
            }
        }
    }

    // ----------------------------------------------------- stability -------
    // evaluateStabilityResidual_ (stability.inc:157-204)
    NZ_HDN void stabilityResidual(int candidate, double P, double T, const double *logRef,
                                      const double *logW, StabilityResidual<NC> &s)
    {
        s.valid = false;
        double maxLogW = logW[0];
#pragma unroll
        for (int i = 1; i < NC; ++i)
            if (maxLogW < logW[i])
                maxLogW = logW[i];
        if (!isfinite(maxLogW))
            return;
        double scaledSum = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double v = exp(logW[i] - maxLogW);
            if (!(v > 0.0) || !isfinite(v))
                return;
            s.x[i] = v;
            scaledSum += v;
        }
        if (!(scaledSum > 0.0) || !isfinite(scaledSum))
            return;
#pragma unroll
        for (int i = 0; i < NC; ++i)
            s.x[i] /= scaledSum;
        const double logSum = maxLogW + log(scaledSum);
        s.sum = logSum > 709.782712893384 ? nzInf() : exp(logSum);
        phase(candidate, P, T, s.x, s.phi);
        s.norm = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double phi = s.phi[i];
            if (!(phi > 0.0) || !isfinite(phi))
                return;
            s.residual[i] = logW[i] + log(phi) - logRef[i];
            s.norm = smax(s.norm, fabs(s.residual[i]));
        }
        s.valid = isfinite(s.norm);
    }

    // evaluateStabilityResidual_ with ln phi from lnPhiMixed (FP32 mixing and
    // fugacity expression, FP64 root; the normalisation of W stays FP64).
    // False when that evaluation fails or the fluid is CPA: the caller then
    // evaluates in FP64.
    NZ_HDN bool stabilityResidualMixed(int candidate, double P, double T, const double *logRef,
                                       const double *logW, StabilityResidual<NC> &s)
    {
        if (F->eosModel == EOS_CPA)
            return false;
        s.valid = false;
        double maxLogW = logW[0];
#pragma unroll
        for (int i = 1; i < NC; ++i)
            if (maxLogW < logW[i])
                maxLogW = logW[i];
        if (!isfinite(maxLogW))
            return false;
        double scaledSum = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double v = exp(logW[i] - maxLogW);
            if (!(v > 0.0) || !isfinite(v))
                return false;
            s.x[i] = v;
            scaledSum += v;
        }
        if (!(scaledSum > 0.0) || !isfinite(scaledSum))
            return false;
#pragma unroll
        for (int i = 0; i < NC; ++i)
            s.x[i] /= scaledSum;
        const double logSum = maxLogW + log(scaledSum);
        s.sum = logSum > 709.782712893384 ? nzInf() : exp(logSum);
        const int role = thermodynamicRole(candidate);
        ensureCache(P, T);
        const MixParams<NC> &p = (role == WATER && sw()) ? aq : nonAq;
        if (!lnPhiMixed<NC>(s.x, p, F->m1, F->m2, role == GAS, s.lnphi))
            return false;
        ++evals;
        s.norm = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            s.residual[i] = logW[i] + s.lnphi[i] - logRef[i];
            s.norm = smax(s.norm, fabs(s.residual[i]));
        }
        s.valid = isfinite(s.norm);
        return s.valid;
    }

    // finalizeStabilityTrial_ (stability.inc:206-223)
    NZ_HD void finalizeTrial(const StabilityResidual<NC> &s, const double *ref, Trial<NC> &t) const
    {
        double dist = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
            dist += fabs(s.x[i] - ref[i]);
        t.valid = true;
        t.trivial = dist < 1.0e-7 && fabs(s.sum - 1.0) < 1.0e-7;
        t.sum = s.sum;
#pragma unroll
        for (int i = 0; i < NC; ++i)
            t.x[i] = s.x[i];
    }

    // stabilityTrial_ (stability.inc:225-355)
    NZ_HDN void stabilityTrial(int candidate, double P, double T, const double *logRef,
                                                const double *ref, const double *seedIn, Trial<NC> &t)
    {
        t.valid = false;
        t.trivial = false;
        t.sum = 0.0;
        double seed[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            seed[i] = seedIn[i];
        normalize(seed);
        double logW[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            logW[i] = log(smax(seed[i], O().floor));
        const int ssiSteps = imin(O().maxStability, imax(O().stabilitySsi, 0));
        StabilityResidual<NC> cur, probe;
#pragma unroll 1
        for (int it = 0; it < ssiSteps; ++it)
        {
            stabilityResidual(candidate, P, T, logRef, logW, cur);
            if (!cur.valid || err)
                return;
            if (cur.norm < O().stabilityTol)
            {
                finalizeTrial(cur, ref, t);
                return;
            }
#pragma unroll
            for (int i = 0; i < NC; ++i)
                logW[i] = logRef[i] - log(smax(cur.phi[i], 1.0e-300));
        }
#pragma unroll 1
        for (int it = 0; it < O().stabilityNewton; ++it)
        {
            stabilityResidual(candidate, P, T, logRef, logW, cur);
            if (!cur.valid || err)
                return;
            if (cur.norm < O().stabilityTol)
            {
                finalizeTrial(cur, ref, t);
                return;
            }
            double J[NC][NC];
#pragma unroll 1
            for (int col = 0; col < NC; ++col)
            {
                double pert[NC];
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    pert[i] = logW[i];
                const double step = O().fdStep * smax(1.0, fabs(logW[col]));
                pert[col] += step;
                stabilityResidual(candidate, P, T, logRef, pert, probe);
                if (!probe.valid)
                    return;
#pragma unroll
                for (int row = 0; row < NC; ++row)
                    J[row][col] = (probe.residual[row] - cur.residual[row]) / step;
            }
            double rhs[NC], delta[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i)
                rhs[i] = -cur.residual[i];
            if (!solveDense<NC>(J, rhs, delta))
                break;
            bool accepted = false;
            double damping = 1.0;
#pragma unroll 1
            for (int ls = 0; ls < 16; ++ls)
            {
                double cand[NC];
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    cand[i] = logW[i] + damping * delta[i];
                stabilityResidual(candidate, P, T, logRef, cand, probe);
                if (probe.valid && probe.norm < cur.norm)
                {
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                        logW[i] = cand[i];
                    accepted = true;
                    break;
                }
                damping *= 0.5;
            }
            if (!accepted)
                break;
        }
        const int remaining = imax(0, O().maxStability - ssiSteps);
#pragma unroll 1
        for (int it = 0; it < remaining; ++it)
        {
            stabilityResidual(candidate, P, T, logRef, logW, cur);
            if (!cur.valid || err)
                return;
            if (cur.norm < O().stabilityTol)
            {
                finalizeTrial(cur, ref, t);
                return;
            }
#pragma unroll
            for (int i = 0; i < NC; ++i)
                logW[i] = logRef[i] - log(smax(cur.phi[i], 1.0e-300));
        }
    }

    // stabilitySeeds_ (stability.inc:32-96): seed k of the candidate list.
    NZ_HD int stabilitySeedCount() const { return NC + 6 + ((F->water >= 0 && NC > 1) ? 1 : 0); }

    NZ_HDN void stabilitySeed(int k, double P, double T, const double *z, const double *ref, double *seed)
    {
        if (k < 4)
        {
            const double exps[4] = {1.0, -1.0, 1.0 / 3.0, -1.0 / 3.0};
            double wilson[NC];
            wilsonK(P, T, wilson);
#pragma unroll
            for (int i = 0; i < NC; ++i)
            {
                const double kk = sclamp(wilson[i], 1.0e-100, 1.0e100);
                seed[i] = z[i] * pow(kk, exps[k]);
            }
            normalize(seed);
            return;
        }
        k -= 4;
        if (k < NC)
        {
            const double remainder = 0.1 / double(NC - 1);
#pragma unroll
            for (int i = 0; i < NC; ++i)
                seed[i] = remainder;
            seed[k] = 0.9;
            return;
        }
        k -= NC;
        if (k == 0 || k == 1)
        {
            const double *src = k == 0 ? z : ref;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                seed[i] = src[i];
            normalize(seed);
            return;
        }
        const double trace = 1.0e-6 / double(NC - 1);
#pragma unroll
        for (int i = 0; i < NC; ++i)
            seed[i] = trace;
        seed[F->water] = 1.0 - 1.0e-6;
    }

    // Lanes hold the first-best trial of their own seeds (seed k on lane
    // k % width); the warp's answer is the largest trial sum, ties going to
    // the lowest seed index -- the sequential loop's first-best rule.  The
    // error flag is shared too, since one failing trial aborts the flash.
    NZ_HD void warpCombineTrials(Trial<NC> &best, int bestK)
    {
#ifdef __CUDA_ARCH__
        __syncwarp();
        int e = err;
        for (int off = 16; off > 0; off >>= 1)
            e = imax(e, __shfl_xor_sync(0xffffffffu, e, off));
        err = e;
        double key = best.valid ? best.sum : -nzInf();
        int kk = best.valid ? bestK : 0x7fffffff;
        for (int off = 16; off > 0; off >>= 1)
        {
            const double ok = __shfl_xor_sync(0xffffffffu, key, off);
            const int ik = __shfl_xor_sync(0xffffffffu, kk, off);
            if (ok > key || (ok == key && ik < kk))
            {
                key = ok;
                kk = ik;
            }
        }
        if (kk == 0x7fffffff)
        {
            best.valid = false;
            return;
        }
        const int src = kk % width;
        best.valid = true;
        best.trivial = __shfl_sync(0xffffffffu, int(best.trivial), src) != 0;
        best.sum = __shfl_sync(0xffffffffu, best.sum, src);
        for (int i = 0; i < NC; ++i)
            best.x[i] = __shfl_sync(0xffffffffu, best.x[i], src);
#else
        (void)best;
        (void)bestK;
#endif
    }

    // stabilityTest (three_phase_flash.hpp:300-489)
    NZ_HDN void stabilityTest(double P, double T, const double *zIn, uint8_t active,
                                               const double (&activeX)[3][NC], StabilityResult<NC> &res)
    {
        res.stable = true;
        res.valid = true;
        res.tested = active;
        for (int p = 0; p < 3; ++p)
        {
            res.unstable[p] = false;
            res.trialSum[p] = 1.0;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                res.incipient[p][i] = 0.0;
        }
        if (stabMemo)
        {
            bool hit = stabMemo->matches(P, T, zIn, active, activeX);
#ifdef __CUDA_ARCH__
            // warp-cooperative lanes take the stored answer together or not at all
            if (width > 1)
                hit = __all_sync(0xffffffffu, hit);
#endif
            if (hit)
            {
                res = stabMemo->res;
                if (stabMemo->err)
                    fail(stabMemo->err);
                return;
            }
        }
        if (!validatePT(P, T))
            return;
        if (active == 0)
        {
            fail(ERR_BAD_INPUT);
            return;
        }
        double z[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            z[i] = zIn[i];
        normalize(z);
        const int ref = firstActive(active);
        double sx[3][NC];
        for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int i = 0; i < NC; ++i)
                sx[p][i] = activeX[p][i];
        if (sw() && popcount3(active) == 1)
#pragma unroll
            for (int i = 0; i < NC; ++i)
                sx[ref][i] = z[i];
        for (int p = 0; p < 3; ++p)
            if (active & bitOf(p))
                normalize(sx[p]);

        if (sw() && popcount3(active) > 1)
        {
            // fugacity-closure certification of the supplied active set (:310-367)
            double phiR[NC], phiP[NC];
            phase(ref, P, T, sx[ref], phiR);
            double mismatch = 0.0;
            for (int p = 0; p < 3; ++p)
            {
                if (!(active & bitOf(p)) || p == ref)
                    continue;
                phase(p, P, T, sx[p], phiP);
#pragma unroll
                for (int i = 0; i < NC; ++i)
                {
                    const double xr = sx[ref][i];
                    const double xp = sx[p][i];
                    if (xr <= 10.0 * O().floor || xp <= 10.0 * O().floor)
                        continue;
                    const double ra = smax(xr * phiR[i], 1.0e-300);
                    const double pa = smax(xp * phiP[i], 1.0e-300);
                    mismatch = smax(mismatch, fabs(log(ra / pa)));
                }
            }
            const double certTol = smax(10.0 * O().fugacityTol, 10.0 * O().stabilityTol);
            if (mismatch > certTol)
            {
                Result<NC> certified;
                flashRestrictedImpl(P, T, z, active, &sx, certified);
                if (!certified.converged || certified.presence != active)
                {
                    res.valid = false;
                    res.stable = false;
                    return;
                }
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                        sx[p][i] = certified.x[p][i];
            }
        }

        double refX[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            refX[i] = sx[ref][i];
        normalize(refX);
        double phiRef[NC];
        phase(ref, P, T, refX, phiRef);
        double logRef[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double xi = smax(refX[i], O().floor);
            const double ph = smax(phiRef[i], 1.0e-300);
            logRef[i] = log(xi) + log(ph);
        }
        const double coincTol = smax(10.0 * O().coincidentTol, 1.0e-7);
        for (int cand = 0; cand < 3; ++cand)
        {
            if (active & bitOf(cand))
                continue;
            Trial<NC> best, trial;
            best.valid = false;
            best.trivial = false;
            best.sum = -nzInf();
            const int nseeds = stabilitySeedCount();
            int bestK = -1;
#pragma unroll 1
            for (int k = lane; k < nseeds; k += width)
            {
                double seed[NC];
                stabilitySeed(k, P, T, z, refX, seed);
                stabilityTrial(cand, P, T, logRef, refX, seed, trial);
                if (trial.valid && (!best.valid || trial.sum > best.sum))
                {
                    best = trial;
                    bestK = k;
                }
                if (err && width == 1)
                    return;
            }
            if (width > 1)
                warpCombineTrials(best, bestK);
            if (err)
                return;
            if (!best.valid)
            {
                res.valid = false;
                res.stable = false;
                continue;
            }
            res.trialSum[cand] = best.sum;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                res.incipient[cand][i] = best.x[i];
            bool coincides = false;
            for (int p = 0; p < 3; ++p)
            {
                if (!(active & bitOf(p)))
                    continue;
                double maxDiff = 0.0;
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    maxDiff = smax(maxDiff, fabs(best.x[i] - sx[p][i]));
                if (maxDiff <= coincTol)
                {
                    coincides = true;
                    break;
                }
            }
            const bool unstable = !best.trivial && !coincides && best.sum > 1.0 + O().stabilityTol;
            res.unstable[cand] = unstable;
            res.stable = res.stable && !unstable;
        }
    }

    // --------------------------------------------------- canonicalisation --
    // refreshCanonicalThermodynamics_ (canonicalization.inc:47-66)
    NZ_HDN void refreshCanonical(double P, double T, Result<NC> &r)
    {
        double phi[NC];
        for (int p = 0; p < 3; ++p)
        {
            if (!(r.presence & bitOf(p)))
                continue;
            normalize(r.x[p]);
            r.Z[p] = phase(p, P, T, r.x[p], phi);
        }
        deriveReferenceK(r);
        updateSaturations(P, T, r);
    }

    // canonicalizeLiquidRoles_ (canonicalization.inc:99-135)
    NZ_HDN void canonicalizeLiquidRoles(Result<NC> &r) const
    {
        if (F->water < 0)
            return;
        const bool hasOil = r.beta[0] > O().betaTol;
        const bool hasWater = r.beta[2] > O().betaTol;
        bool swap = false;
        if (hasOil && hasWater)
        {
            swap = r.x[0][F->water] > r.x[2][F->water];
        }
        else if (hasOil != hasWater)
        {
            const int act = hasOil ? 0 : 2;
            const bool shouldBeWater = waterIsDominant(r.x[act]);
            swap = (hasOil && shouldBeWater) || (hasWater && !shouldBeWater);
        }
        if (swap)
            swapSlots(r, 0, 2);
    }

    // canonicalize_ (canonicalization.inc:8-45)
    NZ_HDN void canonicalize(double P, double T, Result<NC> &r)
    {
        uint8_t p = presenceFromFractions(r.beta);
        if (p == 0)
            p = r.presence == 0 ? OIL_BIT : r.presence;
        r.presence = p;
        double sum = 0.0;
        for (int i = 0; i < 3; ++i)
        {
            double &beta = r.beta[i];
            if (!(p & bitOf(i)) || beta <= O().betaTol || !isfinite(beta))
            {
                beta = 0.0;
                r.presence &= uint8_t(~bitOf(i));
            }
            else
            {
                sum += beta;
            }
        }
        if (!(sum > 0.0))
        {
            r.presence = chooseSinglePhase(P, T, r.x[0]);
            r.beta[0] = r.beta[1] = r.beta[2] = 0.0;
            r.beta[firstActive(r.presence)] = 1.0;
        }
        else
        {
            for (int i = 0; i < 3; ++i)
                r.beta[i] /= sum;
        }
        if (!sw())
            canonicalizeLiquidRoles(r);
        r.presence = presenceFromFractions(r.beta);
        refreshCanonical(P, T, r);
    }

    // canonicalizeGlobalWaterRole_ (canonicalization.inc:175-224)
    NZ_HDN int canonicalizeGlobalWaterRole(Result<NC> &r) const
    {
        if (F->water < 0)
            return -1;
        const int wc = F->water;
        int richest = 2;
        double richestWater = -1.0;
        int activeCount = 0;
        bool hasWaterSlot = false;
        for (int s = 0; s < 3; ++s)
        {
            if (!(r.beta[s] > O().betaTol))
                continue;
            ++activeCount;
            if (s == 2)
                hasWaterSlot = true;
            const double xw = r.x[s][wc];
            if (xw > richestWater)
            {
                richestWater = xw;
                richest = s;
            }
        }
        if (activeCount == 0 || richest == 2)
            return -1;
        if (!hasWaterSlot && !waterIsDominant(r.x[richest]))
            return -1;
        const double currentWater = hasWaterSlot ? r.x[2][wc] : -1.0;
        if (hasWaterSlot && richestWater <= currentWater + 1.0e-10 * smax(1.0, fabs(richestWater)))
            return -1;
        swapSlots(r, richest, 2);
        return richest;
    }

    // validatePhysicalFlashResult_ (canonicalization.inc:225-321)
    NZ_HDN bool validatePhysical(double P, double T, const double *z, const Result<NC> &r)
    {
        if (!r.converged)
            return false;
        const double tol = smax3(10.0 * O().fugacityTol, 10.0 * O().rrTol, 1.0e-10);
        double betaSum = 0.0;
        uint8_t active = 0;
        for (int p = 0; p < 3; ++p)
        {
            const double beta = r.beta[p];
            if (!isfinite(beta) || beta < -tol)
                return false;
            if (beta > O().betaTol)
            {
                active |= uint8_t(bitOf(p));
                betaSum += beta;
                double xsum = 0.0;
#pragma unroll
                for (int i = 0; i < NC; ++i)
                {
                    const double xv = r.x[p][i];
                    if (!isfinite(xv) || xv < -tol)
                        return false;
                    xsum += xv;
                }
                if (fabs(xsum - 1.0) > tol)
                    return false;
            }
        }
        if (active == 0 || fabs(betaSum - 1.0) > tol)
            return false;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            double rec = 0.0;
            for (int p = 0; p < 3; ++p)
                if (active & bitOf(p))
                    rec += r.beta[p] * r.x[p][i];
            if (fabs(rec - z[i]) > tol)
                return false;
        }
        if (popcount3(active) <= 1)
            return true;
        const int ref = firstActive(active);
        double phiR[NC], phiP[NC];
        phaseForRole(ref, P, T, r.x[ref], phiR);
        for (int p = 0; p < 3; ++p)
        {
            if (!(active & bitOf(p)) || p == ref)
                continue;
            phaseForRole(p, P, T, r.x[p], phiP);
#pragma unroll
            for (int i = 0; i < NC; ++i)
            {
                if (r.x[ref][i] <= 10.0 * O().floor || r.x[p][i] <= 10.0 * O().floor)
                    continue;
                const double ra = smax(r.x[ref][i] * phiR[i], 1.0e-300);
                const double pa = smax(r.x[p][i] * phiP[i], 1.0e-300);
                if (fabs(log(ra / pa)) > 10.0 * O().fugacityTol)
                    return false;
            }
        }
        return true;
    }

    // overallComposition_ (canonicalization.inc:323-337)
    NZ_HDN void overallComposition(const Result<NC> &r, double *z)
    {
#pragma unroll
        for (int i = 0; i < NC; ++i)
            z[i] = 0.0;
        for (int s = 0; s < 3; ++s)
        {
            const double beta = r.beta[s];
            if (!(beta > O().betaTol))
                continue;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                z[i] += beta * r.x[s][i];
        }
        normalize(z);
    }

    // reequilibrateCanonicalRoles_ (canonicalization.inc:339-377)
    NZ_HDN void reequilibrateCanonicalRoles(double P, double T, const double *z, Result<NC> &seed,
                                                Result<NC> &out)
    {
        seed.presence = presenceFromFractions(seed.beta);
        const int count = popcount3(seed.presence);
        if (count <= 1)
        {
            singlePhaseResult(P, T, z, seed.presence, out);
            return;
        }
        if (count == 2)
        {
            int first, second;
            activePair(seed.presence, first, second);
            double K[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i)
                K[i] = sclamp(seed.x[second][i] / smax(seed.x[first][i], O().floor), 1.0e-100, 1.0e100);
            flashTwo(P, T, z, first, second, K, out);
            return;
        }
        deriveReferenceK(seed);
        flashThree(P, T, z, seed.Kg, seed.Kw, out);
        if (out.converged)
            return;
        double kg[NC], kw[NC];
        wilsonK(P, T, kg);
        initialWaterK(kw);
        flashThree(P, T, z, kg, kw, out);
    }

    // canonicalizeNonAqueousRoles_ (canonicalization.inc:379-414)
    NZ_HDN bool canonicalizeNonAqueousRoles(double P, double T, Result<NC> &r) const
    {
        const bool hasOil = r.beta[0] > O().betaTol;
        const bool hasGas = r.beta[1] > O().betaTol;
        if (!(hasOil && hasGas))
            return false;
        double wilson[NC];
        wilsonK(P, T, wilson);
        double orientation = 0.0, magnitude = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double lnK = log(sclamp(wilson[i], 1.0e-30, 1.0e30));
            const double term = (r.x[1][i] - r.x[0][i]) * lnK;
            orientation += term;
            magnitude += fabs(term);
        }
        if (orientation >= -1.0e-10 * smax(1.0, magnitude))
            return false;
        swapSlots(r, 0, 1);
        return true;
    }

    // expectedSingleNonAqueousRole_ (canonicalization.inc:416-439)
    NZ_HDN int expectedSingleNonAqueousRole(double P, double T, const double *x) const
    {
        double wilson[NC];
        wilsonK(P, T, wilson);
        double volatility = 0.0, magnitude = 0.0;
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double term = x[i] * log(sclamp(wilson[i], 1.0e-30, 1.0e30));
            volatility += term;
            magnitude += fabs(term);
        }
        return volatility >= -1.0e-10 * smax(1.0, magnitude) ? GAS : OIL;
    }

    // canonicalizeSingleNonAqueousRole_ (canonicalization.inc:441-463)
    NZ_HDN bool canonicalizeSingleNonAqueousRole(double P, double T, Result<NC> &r) const
    {
        const bool hasOil = r.beta[0] > O().betaTol;
        const bool hasGas = r.beta[1] > O().betaTol;
        if (hasOil == hasGas)
            return false;
        const int act = hasOil ? 0 : 1;
        const int expected = expectedSingleNonAqueousRole(P, T, r.x[act]);
        if (act == expected)
            return false;
        swapSlots(r, act, expected);
        r.presence = presenceFromFractions(r.beta);
        return true;
    }

    // canonicalizeCoalescedSwSingleNonAqueousRole_ (canonicalization.inc:466-498)
    NZ_HDN void canonicalizeCoalescedSwSingle(double P, double T, Result<NC> &r)
    {
        if (!sw())
            return;
        const bool hasOil = r.beta[0] > O().betaTol;
        const bool hasGas = r.beta[1] > O().betaTol;
        if (hasOil == hasGas)
            return;
        const int act = hasOil ? 0 : 1;
        double phi[NC];
        const double zo = phaseForRole(OIL, P, T, r.x[act], phi);
        const double zg = phaseForRole(GAS, P, T, r.x[act], phi);
        const double scale = smax3(1.0, fabs(zo), fabs(zg));
        if (fabs(zo - zg) > 1.0e-8 * scale)
            return;
        (void)canonicalizeSingleNonAqueousRole(P, T, r);
    }

    // collapseCoincidentSwPhases_ (canonicalization.inc:507-586)
    NZ_HDN void collapseCoincidentSw(double P, double T, Result<NC> &r)
    {
        if (!sw() || !(O().coincidentTol > 0.0))
            return;
        const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        bool changed = false;
        for (int pass = 0; pass < 2; ++pass)
        {
            bool merged = false;
            for (int k = 0; k < 3; ++k)
            {
                const int a = pairs[k][0], b = pairs[k][1];
                const double betaA = r.beta[a], betaB = r.beta[b];
                if (!(betaA > O().betaTol) || !(betaB > O().betaTol))
                    continue;
                double maxDiff = 0.0;
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    maxDiff = smax(maxDiff, fabs(r.x[a][i] - r.x[b][i]));
                if (maxDiff > O().coincidentTol)
                    continue;
                const double combinedBeta = betaA + betaB;
                double combined[NC];
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    combined[i] = (betaA * r.x[a][i] + betaB * r.x[b][i]) / combinedBeta;
                int dest = a;
                if (a == 2 || b == 2)
                    dest = 2;
                else
                    dest = expectedSingleNonAqueousRole(P, T, combined);
                const int src = dest == a ? b : a;
                r.beta[dest] = combinedBeta;
                r.beta[src] = 0.0;
#pragma unroll
                for (int i = 0; i < NC; ++i)
                {
                    r.x[dest][i] = combined[i];
                    r.x[src][i] = combined[i];
                }
                r.sat[src] = 0.0;
                r.rho[src] = 0.0;
                r.Z[src] = 1.0;
                merged = true;
                changed = true;
                break;
            }
            if (!merged)
                break;
        }
        if (!changed)
            return;
        r.presence = presenceFromFractions(r.beta);
        refreshCanonical(P, T, r);
    }

    // swThermodynamicRolesConsistent_ (canonicalization.inc:588-686)
    NZ_HDN bool swRolesConsistent(double P, double T, const Result<NC> &r, bool preserveRestricted)
    {
        if (!sw() || F->water < 0)
            return true;
        const int wc = F->water;
        int activeCount = 0, aqueousSlot = -1, oilSlot = -1, gasSlot = -1, richestSlot = -1;
        double richestWater = -1.0;
        for (int s = 0; s < 3; ++s)
        {
            if (!(r.beta[s] > O().betaTol))
                continue;
            ++activeCount;
            const int role = roles[s];
            if (role == WATER) aqueousSlot = s;
            if (role == OIL) oilSlot = s;
            if (role == GAS) gasSlot = s;
            const double xw = r.x[s][wc];
            if (xw > richestWater)
            {
                richestWater = xw;
                richestSlot = s;
            }
        }
        if (activeCount == 0)
            return false;
        if (aqueousSlot >= 0)
        {
            if (richestSlot != aqueousSlot &&
                richestWater > r.x[aqueousSlot][wc] + 1.0e-10 * smax(1.0, fabs(richestWater)))
                return false;
        }
        else if (richestSlot >= 0 && waterIsDominant(r.x[richestSlot]))
        {
            return false;
        }
        if ((oilSlot >= 0) != (gasSlot >= 0))
        {
            const int slot = oilSlot >= 0 ? oilSlot : gasSlot;
            const double *x = r.x[slot];
            bool coalesced = false;
            if (preserveRestricted)
            {
                double phi[NC];
                const double zo = phaseForRole(OIL, P, T, x, phi);
                const double zg = phaseForRole(GAS, P, T, x, phi);
                const double scale = smax3(1.0, fabs(zo), fabs(zg));
                coalesced = fabs(zo - zg) <= 1.0e-8 * scale;
            }
            if (!coalesced)
            {
                double pseudoTc = 0.0;
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    pseudoTc += x[i] * F->tc[i];
                const double scale = smax3(1.0, fabs(T), fabs(pseudoTc));
                if (fabs(T - pseudoTc) > 1.0e-8 * scale)
                {
                    const int expected = T > pseudoTc ? GAS : OIL;
                    if (roles[slot] != expected)
                        return false;
                }
            }
        }
        return true;
    }

    // canonicalizeSwThermodynamicRoles_ (canonicalization.inc:688-712)
    NZ_HDN void canonicalizeSwRoles(Result<NC> &r) const
    {
        Result<NC> c = r;
        for (int p = 0; p < 3; ++p)
        {
            c.beta[p] = 0.0;
            c.sat[p] = 0.0;
            c.Z[p] = 1.0;
            c.rho[p] = 0.0;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                c.x[p][i] = 0.0;
        }
        for (int s = 0; s < 3; ++s)
        {
            const int phys = roles[s];
            c.beta[phys] = r.beta[s];
            c.sat[phys] = r.sat[s];
            c.Z[phys] = r.Z[s];
            c.rho[phys] = r.rho[s];
#pragma unroll
            for (int i = 0; i < NC; ++i)
                c.x[phys][i] = r.x[s][i];
        }
        c.presence = presenceFromFractions(c.beta);
        deriveReferenceK(c);
        r = c;
    }

    // canonicalizeFinal_ (canonicalization.inc:714-796)
    NZ_HDN void canonicalizeFinal(double P, double T, Result<NC> &r, bool preserveRestricted)
    {
        if (!r.converged)
            return;
        if (sw())
        {
            if (!swRolesConsistent(P, T, r, preserveRestricted))
            {
                r.converged = false;
                return;
            }
            canonicalizeSwRoles(r);
            collapseCoincidentSw(P, T, r);
            if (!preserveRestricted)
                canonicalizeCoalescedSwSingle(P, T, r);
            (void)canonicalizeNonAqueousRoles(P, T, r);
            r.presence = presenceFromFractions(r.beta);
            return;
        }
        for (int pass = 0; pass < 4; ++pass)
        {
            r.presence = presenceFromFractions(r.beta);
            double z[NC];
            overallComposition(r, z);
            const int waterSource = canonicalizeGlobalWaterRole(r);
            const bool crossedGasWater = waterSource == GAS;
            const bool crossedSingle = !preserveRestricted && canonicalizeSingleNonAqueousRole(P, T, r);
            if (crossedGasWater || crossedSingle)
            {
                r.presence = presenceFromFractions(r.beta);
                Result<NC> corrected;
                reequilibrateCanonicalRoles(P, T, z, r, corrected);
                if (!corrected.converged)
                {
                    r.converged = false;
                    return;
                }
                r = corrected;
                continue;
            }
            (void)canonicalizeNonAqueousRoles(P, T, r);
            r.presence = presenceFromFractions(r.beta);
            refreshCanonical(P, T, r);
            return;
        }
        r.converged = false;
    }


    // ------------------------------------------- SW allocation recovery ----
    // evaluateAllocation_ (allocation.inc:31-128): softmax allocation u -> state
    struct AllocState
    {
        bool valid;
        double gibbs;
        double closure;
        double residualNorm2;
        double residual[2 * NC];
        double gradient[2 * NC];
        double x[3][NC];
        double beta[3];
        double Z[3];
    };

    NZ_HDN void evaluateAllocation(double P, double T, const double *z, const double *u, AllocState &s)
    {
        s.valid = false;
        s.gibbs = 0.0;
        s.closure = nzInf();
        s.residualNorm2 = nzInf();
        s.beta[0] = s.beta[1] = s.beta[2] = 0.0;
        double amount[3][NC];
#pragma unroll 1
        for (int c = 0; c < NC; ++c)
        {
            const double ug = u[c];
            const double uw = u[NC + c];
            const double shift = smax3(0.0, ug, uw);
            const double qo0 = exp(-shift);
            const double qg0 = exp(ug - shift);
            const double qw0 = exp(uw - shift);
            const double qsum = qo0 + qg0 + qw0;
            const double qo = qo0 / qsum, qg = qg0 / qsum, qw = qw0 / qsum;
            amount[0][c] = z[c] * qo;
            amount[1][c] = z[c] * qg;
            amount[2][c] = z[c] * qw;
            s.beta[0] += amount[0][c];
            s.beta[1] += amount[1][c];
            s.beta[2] += amount[2][c];
        }
        for (int p = 0; p < 3; ++p)
        {
            if (!(s.beta[p] > 1.0e-14))
                return;
#pragma unroll 1
            for (int c = 0; c < NC; ++c)
                s.x[p][c] = amount[p][c] / s.beta[p];
        }
        double mu[3][NC];
        double phi[NC];
        for (int p = 0; p < 3; ++p)
        {
            s.Z[p] = phase(p, P, T, s.x[p], phi);
#pragma unroll 1
            for (int c = 0; c < NC; ++c)
            {
                const double xv = smax(s.x[p][c], O().floor);
                const double ph = smax(phi[c], 1.0e-300);
                mu[p][c] = log(xv) + log(ph);
                s.gibbs += amount[p][c] * mu[p][c];
            }
        }
        s.closure = 0.0;
        s.residualNorm2 = 0.0;
#pragma unroll 1
        for (int c = 0; c < NC; ++c)
        {
            const int w = NC + c;
            if (!(z[c] > O().floor))
            {
                s.residual[c] = s.residual[w] = 0.0;
                s.gradient[c] = s.gradient[w] = 0.0;
                continue;
            }
            s.residual[c] = mu[1][c] - mu[0][c];
            s.residual[w] = mu[2][c] - mu[0][c];
            s.residualNorm2 += s.residual[c] * s.residual[c] + s.residual[w] * s.residual[w];
            double cl = s.closure;
            const double d01 = fabs(mu[0][c] - mu[1][c]);
            const double d02 = fabs(mu[0][c] - mu[2][c]);
            const double d12 = fabs(mu[1][c] - mu[2][c]);
            if (cl < d01) cl = d01;
            if (cl < d02) cl = d02;
            if (cl < d12) cl = d12;
            s.closure = cl;
            const double qo = amount[0][c] / z[c];
            const double qg = amount[1][c] / z[c];
            const double qw = amount[2][c] / z[c];
            const double average = qo * mu[0][c] + qg * mu[1][c] + qw * mu[2][c];
            s.gradient[c] = z[c] * qg * (mu[1][c] - average);
            s.gradient[w] = z[c] * qw * (mu[2][c] - average);
        }
        s.valid = isfinite(s.gibbs) && isfinite(s.residualNorm2) && isfinite(s.closure);
    }

    // gibbsPreconditionAllocation_ (allocation.inc:134-239): BFGS on the Gibbs energy
    NZ_HDN void gibbsPrecondition(double P, double T, const double *z, double *u, AllocState &state)
    {
        constexpr int M = 2 * NC;
        double H[M][M];
        for (int i = 0; i < M; ++i)
            for (int j = 0; j < M; ++j)
                H[i][j] = i == j ? 1.0 : 0.0;
        evaluateAllocation(P, T, z, u, state);
        if (!state.valid)
            return;
        AllocState trial;
#pragma unroll 1
        for (int it = 0; it < 160; ++it)
        {
            if (err)
                return;
            double dir[M];
            for (int i = 0; i < M; ++i)
            {
                dir[i] = 0.0;
                for (int j = 0; j < M; ++j)
                    dir[i] -= H[i][j] * state.gradient[j];
            }
            double dd = 0.0, maxStep = 0.0;
            for (int i = 0; i < M; ++i)
            {
                dd += state.gradient[i] * dir[i];
                maxStep = smax(maxStep, fabs(dir[i]));
            }
            if (!(dd < 0.0) || !isfinite(dd))
            {
                dd = 0.0;
                maxStep = 0.0;
                for (int i = 0; i < M; ++i)
                {
                    for (int j = 0; j < M; ++j)
                        H[i][j] = i == j ? 1.0 : 0.0;
                    dir[i] = -state.gradient[i];
                    dd += state.gradient[i] * dir[i];
                    maxStep = smax(maxStep, fabs(dir[i]));
                }
            }
            if (maxStep > 4.0)
                for (int i = 0; i < M; ++i)
                    dir[i] *= 4.0 / maxStep;
            double trialU[M];
            double step = 1.0;
            bool accepted = false;
#pragma unroll 1
            for (int ls = 0; ls < 24; ++ls)
            {
                for (int i = 0; i < M; ++i)
                    trialU[i] = sclamp(u[i] + step * dir[i], -40.0, 40.0);
                evaluateAllocation(P, T, z, trialU, trial);
                if (trial.valid && trial.gibbs <= state.gibbs + 1.0e-4 * step * dd)
                {
                    accepted = true;
                    break;
                }
                step *= 0.5;
            }
            if (!accepted)
                return;
            double sv[M], yv[M], hy[M];
            double ys = 0.0;
            for (int i = 0; i < M; ++i)
            {
                sv[i] = trialU[i] - u[i];
                yv[i] = trial.gradient[i] - state.gradient[i];
            }
            for (int i = 0; i < M; ++i)
                ys += yv[i] * sv[i];
            if (ys > 1.0e-12)
            {
                for (int i = 0; i < M; ++i)
                {
                    hy[i] = 0.0;
                    for (int j = 0; j < M; ++j)
                        hy[i] += H[i][j] * yv[j];
                }
                double yhy = 0.0;
                for (int i = 0; i < M; ++i)
                    yhy += yv[i] * hy[i];
                const double coef = (ys + yhy) / (ys * ys);
                for (int i = 0; i < M; ++i)
                    for (int j = 0; j < M; ++j)
                        H[i][j] += coef * sv[i] * sv[j] - (hy[i] * sv[j] + sv[i] * hy[j]) / ys;
            }
            else
            {
                for (int i = 0; i < M; ++i)
                    for (int j = 0; j < M; ++j)
                        H[i][j] = i == j ? 1.0 : 0.0;
            }
            for (int i = 0; i < M; ++i)
                u[i] = trialU[i];
            state = trial;
        }
    }

    // refineAllocationChemicalPotentials_ (allocation.inc:246-346): LM on mu differences
    NZ_HDN bool refineAllocation(double P, double T, const double *z, double *u, AllocState &state)
    {
        constexpr int M = 2 * NC;
        evaluateAllocation(P, T, z, u, state);
        if (!state.valid)
            return false;
        double lambda = 1.0e-5;
        AllocState ps, ms, trial;
        double J[M][M];
#pragma unroll 1
        for (int it = 0; it < 160; ++it)
        {
            if (err)
                return false;
            if (state.closure < O().fugacityTol)
                return true;
#pragma unroll 1
            for (int col = 0; col < M; ++col)
            {
                const double h = 2.0e-5 * smax(1.0, fabs(u[col]));
                double plus[M], minus[M];
                for (int i = 0; i < M; ++i)
                    plus[i] = minus[i] = u[i];
                plus[col] = smin(40.0, u[col] + h);
                minus[col] = smax(-40.0, u[col] - h);
                evaluateAllocation(P, T, z, plus, ps);
                evaluateAllocation(P, T, z, minus, ms);
                if (!ps.valid || !ms.valid)
                    return false;
                const double den = plus[col] - minus[col];
                for (int row = 0; row < M; ++row)
                    J[row][col] = (ps.residual[row] - ms.residual[row]) / den;
            }
            bool accepted = false;
#pragma unroll 1
            for (int lm = 0; lm < 14 && !accepted; ++lm)
            {
                double Nm[M][M], rhs[M], delta[M];
                for (int a = 0; a < M; ++a)
                {
                    for (int b = 0; b < M; ++b)
                    {
                        double v = 0.0;
                        for (int row = 0; row < M; ++row)
                            v += J[row][a] * J[row][b];
                        Nm[a][b] = v;
                    }
                    double v = 0.0;
                    for (int row = 0; row < M; ++row)
                        v += J[row][a] * state.residual[row];
                    rhs[a] = -v;
                    Nm[a][a] += lambda;
                }
                if (!solveDense<M>(Nm, rhs, delta))
                {
                    lambda *= 10.0;
                    continue;
                }
                double maxDelta = 0.0;
                for (int i = 0; i < M; ++i)
                    maxDelta = smax(maxDelta, fabs(delta[i]));
                if (maxDelta > 6.0)
                    for (int i = 0; i < M; ++i)
                        delta[i] *= 6.0 / maxDelta;
                double damping = 1.0;
#pragma unroll 1
                for (int ls = 0; ls < 22; ++ls)
                {
                    double trialU[M];
                    for (int i = 0; i < M; ++i)
                        trialU[i] = sclamp(u[i] + damping * delta[i], -40.0, 40.0);
                    evaluateAllocation(P, T, z, trialU, trial);
                    if (trial.valid && trial.residualNorm2 < state.residualNorm2 * (1.0 - 1.0e-5 * damping))
                    {
                        for (int i = 0; i < M; ++i)
                            u[i] = trialU[i];
                        state = trial;
                        lambda = smax(1.0e-14, lambda * 0.2);
                        accepted = true;
                        break;
                    }
                    damping *= 0.5;
                }
                if (!accepted)
                    lambda *= 10.0;
            }
            if (!accepted)
                return false;
        }
        return state.closure < O().fugacityTol;
    }

    // amounts -> allocation variables (shared tail of the seed builders)
    NZ_HD void allocationFromAmounts(const double *z, const double (&amount)[3][NC], double *u) const
    {
        for (int c = 0; c < NC; ++c)
        {
            if (!(z[c] > O().floor))
            {
                u[c] = 0.0;
                u[NC + c] = 0.0;
                continue;
            }
            const double qo = smax(amount[0][c] / z[c], 1.0e-18);
            const double qg = smax(amount[1][c] / z[c], 1.0e-18);
            const double qw = smax(amount[2][c] / z[c], 1.0e-18);
            u[c] = log(qg / qo);
            u[NC + c] = log(qw / qo);
        }
    }

    // allocationSeedFromPair_ (allocation.inc:361-446)
    NZ_HDN bool allocationSeedFromPair(double P, double T, const double *z, uint8_t allowed, double *u)
    {
        Result<NC> pair;
        flashRestrictedRecovery(P, T, z, allowed, pair);
        if (!pair.converged || popcount3(pair.presence) != 2)
            return false;
        StabilityResult<NC> st;
        stabilityTest(P, T, z, pair.presence, pair.x, st);
        int missing = -1;
        for (int p = 0; p < 3; ++p)
            if (!(pair.presence & bitOf(p)))
            {
                missing = p;
                break;
            }
        if (missing < 0 || !st.valid || !st.unstable[missing])
            return false;
        const double *inc = st.incipient[missing];
        double eps = 1.0e-3;
        for (int c = 0; c < NC; ++c)
            if (inc[c] > 1.0e-30)
                eps = smin(eps, 0.15 * z[c] / inc[c]);
        eps = smax(eps, 1.0e-9);
        double amount[3][NC];
        for (int p = 0; p < 3; ++p)
            for (int c = 0; c < NC; ++c)
                amount[p][c] = 0.0;
        for (int c = 0; c < NC; ++c)
        {
            if (!(z[c] > O().floor))
                continue;
            amount[missing][c] = eps * inc[c];
            const double remaining = z[c] - amount[missing][c];
            if (!(remaining > 0.0))
                return false;
            double pairAmount = 0.0;
            for (int p = 0; p < 3; ++p)
                if (p != missing)
                    pairAmount += pair.beta[p] * pair.x[p][c];
            if (!(pairAmount > 0.0))
                return false;
            for (int p = 0; p < 3; ++p)
                if (p != missing)
                    amount[p][c] = pair.beta[p] * pair.x[p][c] * remaining / pairAmount;
        }
        allocationFromAmounts(z, amount, u);
        return true;
    }

    // allocationSeedFromRawOg_ (allocation.inc:449-502)
    NZ_HDN bool allocationSeedFromRawOg(double P, double T, const double *z, double *u)
    {
        double kg[NC];
        wilsonK(P, T, kg);
        Result<NC> pair;
        flashTwo(P, T, z, OIL, GAS, kg, pair);
        if (!pair.converged || popcount3(presenceFromFractions(pair.beta)) != 2)
            return false;
        pair.presence = presenceFromFractions(pair.beta);
        StabilityResult<NC> st;
        stabilityTest(P, T, z, pair.presence, pair.x, st);
        if (!st.valid || !st.unstable[WATER])
            return false;
        const double *inc = st.incipient[WATER];
        double eps = 1.0e-3;
        for (int c = 0; c < NC; ++c)
            if (inc[c] > 1.0e-30)
                eps = smin(eps, 0.2 * z[c] / inc[c]);
        eps = smax(eps, 1.0e-9);
        double amount[3][NC];
        for (int c = 0; c < NC; ++c)
        {
            if (!(z[c] > O().floor))
            {
                u[c] = 0.0;
                u[NC + c] = 0.0;
                continue;
            }
            amount[2][c] = eps * inc[c];
            const double remaining = z[c] - amount[2][c];
            const double no = pair.beta[0] * pair.x[0][c];
            const double ng = pair.beta[1] * pair.x[1][c];
            const double sum = no + ng;
            if (!(remaining > 0.0) || !(sum > 0.0))
                return false;
            amount[0][c] = no * remaining / sum;
            amount[1][c] = ng * remaining / sum;
            const double qo = smax(amount[0][c] / z[c], 1.0e-18);
            const double qg = smax(amount[1][c] / z[c], 1.0e-18);
            const double qw = smax(amount[2][c] / z[c], 1.0e-18);
            u[c] = log(qg / qo);
            u[NC + c] = log(qw / qo);
        }
        return true;
    }

    // allocationSeedFromSingle_ (allocation.inc:504-578)
    NZ_HDN bool allocationSeedFromSingle(double P, double T, const double *z, double *u)
    {
        const uint8_t active = chooseSinglePhase(P, T, z);
        Result<NC> single;
        singlePhaseResult(P, T, z, active, single);
        StabilityResult<NC> st;
        stabilityTest(P, T, z, active, single.x, st);
        if (!st.valid || st.stable)
            return false;
        double eps[3] = {0.0, 0.0, 0.0};
        int missingCount = 0;
        for (int p = 0; p < 3; ++p)
            if (!(active & bitOf(p)) && st.unstable[p])
            {
                eps[p] = 1.0e-4;
                ++missingCount;
            }
        if (missingCount == 0)
            return false;
        for (int c = 0; c < NC; ++c)
            for (int p = 0; p < 3; ++p)
            {
                if (!(eps[p] > 0.0))
                    continue;
                eps[p] = smin(eps[p], 0.08 * z[c] / smax(st.incipient[p][c], 1.0e-30));
            }
        double amount[3][NC];
        for (int p = 0; p < 3; ++p)
            for (int c = 0; c < NC; ++c)
                amount[p][c] = 0.0;
        const int activeSlot = firstActive(active);
        for (int c = 0; c < NC; ++c)
        {
            if (!(z[c] > O().floor))
            {
                u[c] = 0.0;
                u[NC + c] = 0.0;
                continue;
            }
            double removed = 0.0;
            for (int p = 0; p < 3; ++p)
            {
                if (!(eps[p] > 0.0))
                    continue;
                amount[p][c] = eps[p] * st.incipient[p][c];
                removed += amount[p][c];
            }
            if (!(z[c] > removed))
                return false;
            amount[activeSlot][c] = z[c] - removed;
            const double qo = smax(amount[0][c] / z[c], 1.0e-18);
            const double qg = smax(amount[1][c] / z[c], 1.0e-18);
            const double qw = smax(amount[2][c] / z[c], 1.0e-18);
            u[c] = log(qg / qo);
            u[NC + c] = log(qw / qo);
        }
        return true;
    }

    // thermodynamicAllocationSeed_ (allocation.inc:581-604)
    NZ_HD void thermodynamicAllocationSeed(double P, double T, double scale, double gs, double ws, double *u) const
    {
        double kg[NC], kw[NC];
        wilsonK(P, T, kg);
        initialWaterK(kw);
        for (int c = 0; c < NC; ++c)
        {
            u[c] = sclamp(scale * log(sclamp(kg[c], 1.0e-30, 1.0e30)) + gs, -30.0, 30.0);
            u[NC + c] = sclamp(scale * log(sclamp(kw[c], 1.0e-30, 1.0e30)) + ws, -30.0, 30.0);
        }
    }

    // One seed of flashThreeAllocationFallback_ (allocation.inc:609-700):
    // build seed k (of 23, in the reference's order), precondition and refine
    // it.  True when it ends in an admissible three-phase allocation (`state`
    // holds it, with its Gibbs energy).
    NZ_HDN bool allocationSeedState(double P, double T, const double *z, int k, AllocState &state)
    {
        const uint8_t pairs[3] = {OIL_BIT | GAS_BIT, OIL_BIT | WATER_BIT, GAS_BIT | WATER_BIT};
        const double thermo[6][3] = {{1.0, 0.0, 0.0}, {0.5, 0.0, 0.0}, {1.5, 0.0, 0.0},
                                     {1.0, -1.5, -1.5}, {1.0, 1.5, -1.5}, {1.0, -1.5, 1.5}};
        const double generic[12][2] = {{0.0, 0.0}, {1.0, -2.0}, {2.0, -4.0}, {2.0, -2.0},
                                       {1.0, -4.0}, {-1.0, -1.0}, {-2.0, -2.0}, {-2.0, 1.0},
                                       {-1.0, 2.0}, {2.0, 1.0}, {1.0, 2.0}, {-2.0, 2.0}};
        double u[2 * NC];
        bool valid = true;
        if (k == 0)
            valid = allocationSeedFromRawOg(P, T, z, u);
        else if (k == 1)
            valid = allocationSeedFromSingle(P, T, z, u);
        else if (k < 5)
            valid = allocationSeedFromPair(P, T, z, pairs[k - 2], u);
        else if (k < 11)
            thermodynamicAllocationSeed(P, T, thermo[k - 5][0], thermo[k - 5][1], thermo[k - 5][2], u);
        else
            for (int c = 0; c < NC; ++c)
            {
                u[c] = generic[k - 11][0];
                u[NC + c] = generic[k - 11][1];
            }
        if (!valid)
            return false;
        gibbsPrecondition(P, T, z, u, state);
        if (!state.valid)
            return false;
        if (!refineAllocation(P, T, z, u, state))
            return false;
        return state.beta[0] > O().betaTol && state.beta[1] > O().betaTol && state.beta[2] > O().betaTol;
    }

    // The three-phase result of an accepted allocation.
    NZ_HDN void allocationCandidate(double P, double T, const double (&beta)[3], const double (&Z)[3],
                                    const double (&x)[3][NC], Result<NC> &cand)
    {
        cand.init();
        cand.converged = true;
        cand.presence = ALL_BITS;
        for (int p = 0; p < 3; ++p)
        {
            cand.beta[p] = beta[p];
            cand.Z[p] = Z[p];
            for (int c = 0; c < NC; ++c)
                cand.x[p][c] = x[p][c];
        }
        deriveReferenceK(cand);
        updateSaturations(P, T, cand);
    }
    NZ_HDN void allocationCandidate(double P, double T, const AllocState &state, Result<NC> &cand)
    {
        allocationCandidate(P, T, state.beta, state.Z, state.x, cand);
    }

    // Seed k's outcome for an AllocMemo (run with width 1; err is left as it was).
    NZ_HDN void allocationSeedOutcome(double P, double T, const double *z, int k, AllocSeedOut<NC> &o)
    {
        const int before = err;
        err = ERR_NONE;
        AllocState state;
        const bool admissible = allocationSeedState(P, T, z, k, state);
        o.err = err;
        err = before;
        o.admissible = admissible ? 1 : 0;
        o.gibbs = admissible ? state.gibbs : 0.0;
        for (int p = 0; p < 3; ++p)
        {
            o.beta[p] = admissible ? state.beta[p] : 0.0;
            o.Z[p] = admissible ? state.Z[p] : 0.0;
            for (int c = 0; c < NC; ++c)
                o.x[p][c] = admissible ? state.x[p][c] : 0.0;
        }
    }

    // The sequential acceptance over stored seed outcomes.  An error of seed
    // k ends the search there (the caller returns on it, so `best` no longer
    // matters).
    NZ_HDN void allocationReplay(double P, double T, const AllocMemo<NC> &m, Result<NC> &best)
    {
        double bestG = nzInf();
        Result<NC> cand;
#pragma unroll 1
        for (int k = 0; k < kAllocationSeeds; ++k)
        {
            if (err)
                return;
            const AllocSeedOut<NC> &o = m.seed[k];
            if (o.err != ERR_NONE)
            {
                fail(o.err);
                return;
            }
            if (!o.admissible || !(o.gibbs < bestG))
                continue;
            allocationCandidate(P, T, o.beta, o.Z, o.x, cand);
            if (!cand.converged)
                continue;
            best = cand;
            bestG = o.gibbs;
        }
    }

    static constexpr int kAllocationSeeds = kAllocSeedCount;

    // flashThreeAllocationFallback_ (allocation.inc:609-700): the seeds in
    // order, a seed replacing the best only with a strictly lower Gibbs
    // energy; the first error ends the search.  The answer is therefore the
    // first seed that reaches the lowest energy among the admissible ones,
    // which lets warp-cooperative lanes run one seed each
    // (allocationFallbackWarp) and reproduce it.
    NZ_HDN void allocationFallback(double P, double T, const double *z, Result<NC> &best)
    {
        best.init();
        if (allocMemo && roles[0] == OIL && roles[1] == GAS && roles[2] == WATER &&
            allocMemo->matches(P, T, salinity, z))
        {
            allocationReplay(P, T, *allocMemo, best);
            return;
        }
#ifdef __CUDA_ARCH__
        if (width > 1)
        {
            allocationFallbackWarp(P, T, z, best);
            return;
        }
#endif
        double bestG = nzInf();
        AllocState state;
        Result<NC> cand;
#pragma unroll 1
        for (int k = 0; k < kAllocationSeeds; ++k)
        {
            if (err)
                return;
            if (!allocationSeedState(P, T, z, k, state))
                continue;
            if (!(state.gibbs < bestG))
                continue;
            allocationCandidate(P, T, state, cand);
            if (!cand.converged)
                continue;
            best = cand;
            bestG = state.gibbs;
        }
    }

#ifdef __CUDA_ARCH__
    // Lane k runs seed k alone (width 1, its own error flag); the warp then
    // replays the sequential acceptance over the seeds' outcomes in order and
    // takes the chosen candidate from its lane.  A candidate's saturation
    // update runs on its lane whether or not the sequential loop would reach
    // it; its error only counts where the loop would have run it.
    NZ_HDN void allocationFallbackWarp(double P, double T, const double *z, Result<NC> &best)
    {
        static_assert(kAllocationSeeds <= 32, "one allocation seed per lane");
        if (err)
            return;
        const int savedWidth = width;
        const int savedLane = lane;
        const unsigned long long evals0 = evals;
        width = 1;
        lane = 0;
        bool admissible = false;
        bool candidateOk = false;
        int seedErr = ERR_NONE;
        int candErr = ERR_NONE;
        double g = 0.0;
        Result<NC> mine;
        mine.init();
        if (savedLane < kAllocationSeeds)
        {
            AllocState state;
            admissible = allocationSeedState(P, T, z, savedLane, state);
            seedErr = err;
            err = ERR_NONE;
            if (admissible && seedErr == ERR_NONE)
            {
                g = state.gibbs;
                allocationCandidate(P, T, state, mine);
                candErr = err;
                err = ERR_NONE;
                candidateOk = mine.converged;
            }
        }
        width = savedWidth;
        lane = savedLane;
        __syncwarp();
        unsigned long long spent = evals - evals0;
        for (int off = 16; off > 0; off >>= 1)
            spent += __shfl_xor_sync(0xffffffffu, spent, off);
        evals = evals0 + spent;
        double bestG = nzInf();
        int bestK = -1;
        int code = ERR_NONE;
#pragma unroll 1
        for (int k = 0; k < kAllocationSeeds; ++k)
        {
            const int ek = __shfl_sync(0xffffffffu, seedErr, k);
            const bool ok = __shfl_sync(0xffffffffu, int(admissible), k) != 0;
            const double gk = __shfl_sync(0xffffffffu, g, k);
            const int ck = __shfl_sync(0xffffffffu, candErr, k);
            const bool conv = __shfl_sync(0xffffffffu, int(candidateOk), k) != 0;
            if (ek != ERR_NONE)
            {
                code = ek;
                break;
            }
            if (!ok || !(gk < bestG))
                continue;
            if (ck != ERR_NONE)
            {
                bestK = k;
                code = ck;
                break;
            }
            if (!conv)
                continue;
            bestK = k;
            bestG = gk;
        }
        if (code != ERR_NONE)
            fail(code);
        if (bestK >= 0)
            shuffleResult(mine, bestK, best);
    }
#endif

    // ------------------------------------------------------- active set ----
    // equilibrateActiveSet_ (allocation.inc:707-858)
    NZ_HDN void equilibrateActiveSet(double P, double T, const double *z, uint8_t active,
                                                      Result<NC> &seed, bool reuseConvergedSeed,
                                                      Result<NC> &out)
    {
        if (active == 0)
            active = chooseSinglePhase(P, T, z);
        canonicalize(P, T, seed);
        if (seed.presence != active)
            active = seed.presence;
        Result<NC> lastPhysical = seed;
        bool useConvergedSeed = reuseConvergedSeed && seed.converged && seed.presence == active && !sw();
        Result<NC> &current = out;
#pragma unroll 1
        for (int outer = 0; outer < 8; ++outer)
        {
            if (err)
            {
                out.converged = false;
                return;
            }
            if (useConvergedSeed)
            {
                current = seed;
                useConvergedSeed = false;
            }
            else if (popcount3(active) == 1)
            {
                singlePhaseResult(P, T, z, active, current);
            }
            else if (popcount3(active) == 2)
            {
                int first, second;
                activePair(active, first, second);
                double K[NC];
                pairInitialK(first, second, P, T, z, K);
                if (seed.converged && seed.presence == active)
                {
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                        K[i] = sclamp(seed.x[second][i] / smax(seed.x[first][i], O().floor),
                                      1.0e-100, 1.0e100);
                }
                flashTwo(P, T, z, first, second, K, current);
                if (!current.converged)
                    singlePhaseResult(P, T, z, chooseSinglePhase(P, T, z), current);
            }
            else
            {
                double kg[NC], kw[NC];
                bool kgValid = true, kwValid = true;
#pragma unroll
                for (int i = 0; i < NC; ++i)
                {
                    kg[i] = seed.Kg[i];
                    kw[i] = seed.Kw[i];
                    kgValid = kgValid && kg[i] > 0.0;
                    kwValid = kwValid && kw[i] > 0.0;
                }
                if (!kgValid) wilsonK(P, T, kg);
                if (!kwValid) initialWaterK(kw);
                flashThree(P, T, z, kg, kw, current);
                if (!current.converged)
                {
                    lastPhysical.converged = false;
                    canonicalize(P, T, lastPhysical);
                    out = lastPhysical;
                    return;
                }
            }

            uint8_t fractionPresence = presenceFromFractions(current.beta);
            if (fractionPresence == 0)
                fractionPresence = chooseSinglePhase(P, T, z);
            if (fractionPresence != active)
            {
                active = fractionPresence;
                seed = current;
                canonicalize(P, T, seed);
                lastPhysical = seed;
                useConvergedSeed = seed.converged && seed.presence == active && !sw();
                continue;
            }
            canonicalize(P, T, current);
            lastPhysical = current;
            if (popcount3(active) == 3)
            {
                canonicalize(P, T, current);
                return;
            }
            StabilityResult<NC> st;
            stabilityTest(P, T, z, active, current.x, st);
            if (!st.valid)
            {
                current.converged = false;
                canonicalize(P, T, current);
                return;
            }
            if (st.stable)
            {
                canonicalize(P, T, current);
                return;
            }
            bool added = false;
            for (int p = 0; p < 3; ++p)
            {
                if (!(active & bitOf(p)) && st.unstable[p])
                {
                    active |= uint8_t(bitOf(p));
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                        seed.x[p][i] = st.incipient[p][i];
                    added = true;
                }
            }
            if (!added)
            {
                current.converged = false;
                canonicalize(P, T, current);
                return;
            }
            deriveReferenceK(seed);
            seed.presence = active;
            useConvergedSeed = false;
        }
        canonicalize(P, T, seed);
        out = seed;
    }

    // ------------------------------------------------- restricted flashes --
    // flashRestrictedImpl_ (restricted.inc:8-59).  A three-phase `allowed`
    // set is never requested by the entry points carried here.
    NZ_HDN void flashRestrictedImpl(double P, double T, const double *zIn, uint8_t allowed,
                                                     const double (*seedX)[3][NC], Result<NC> &r)
    {
        r.init();
        if (!validatePT(P, T))
            return;
        double z[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            z[i] = zIn[i];
        normalize(z);
        if (allowed == 0)
        {
            fail(ERR_BAD_INPUT);
            return;
        }
        if (popcount3(allowed) == 3)
        {
            fail(ERR_NOT_PORTED);
            return;
        }
        if (popcount3(allowed) == 1)
        {
            singlePhaseResult(P, T, z, allowed, r);
            return;
        }
        int first, second;
        activePair(allowed, first, second);
        double K[NC];
        pairInitialK(first, second, P, T, z, K);
        if (seedX != nullptr)
        {
            double a[NC], b[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i)
            {
                a[i] = (*seedX)[first][i];
                b[i] = (*seedX)[second][i];
            }
            normalize(a);
            normalize(b);
#pragma unroll
            for (int i = 0; i < NC; ++i)
                K[i] = sclamp(b[i] / smax(a[i], O().floor), 1.0e-100, 1.0e100);
        }
        flashTwo(P, T, z, first, second, K, r);
        if (!r.converged && seedX != nullptr)
        {
            pairInitialK(first, second, P, T, z, K);
            flashTwo(P, T, z, first, second, K, r);
        }
        if (r.converged)
            canonicalize(P, T, r);
    }

    // flashRestricted (three_phase_flash.hpp:235-292), both overloads
    NZ_HDN void flashRestricted(double P, double T, const double *zIn, uint8_t allowed,
                                                 const double (*seedX)[3][NC], Result<NC> &r)
    {
        double z[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            z[i] = zIn[i];
        normalize(z);
        flashRestrictedImpl(P, T, z, allowed, seedX, r);
        if (!r.converged && popcount3(allowed) == 2 && sw())
        {
            int first, second;
            activePair(allowed, first, second);
            finalizePhysicallyConvergedTwoPhase(P, T, z, first, second, r);
        }
        if (r.converged)
        {
            canonicalizeFinal(P, T, r, true);
            if (r.converged && !validatePhysical(P, T, z, r))
                r.converged = false;
        }
    }

    // flashRestrictedRecovery_ (restricted.inc:629-646)
    NZ_HDN void flashRestrictedRecovery(double P, double T, const double *zIn, uint8_t allowed, Result<NC> &r)
    {
        double z[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            z[i] = zIn[i];
        normalize(z);
        flashRestrictedImpl(P, T, z, allowed, nullptr, r);
        if (r.converged)
        {
            canonicalizeFinal(P, T, r, false);
            if (r.converged && !validatePhysical(P, T, z, r))
                r.converged = false;
        }
    }

    // stableReducedSetFallback_ (restricted.inc:655-693)
    NZ_HDN void stableReducedSetFallback(double P, double T, const double *z, Result<NC> &best)
    {
        best.init();
        double bestG = nzInf();
        const uint8_t pairs[3] = {OIL_BIT | GAS_BIT, OIL_BIT | WATER_BIT, GAS_BIT | WATER_BIT};
        Result<NC> cand;
        for (int k = 0; k < 3; ++k)
        {
            flashRestrictedRecovery(P, T, z, pairs[k], cand);
            if (err)
                return;
            if (!cand.converged)
                continue;
            cand.presence = presenceFromFractions(cand.beta);
            if (cand.presence == 0)
                continue;
            StabilityResult<NC> st;
            stabilityTest(P, T, z, cand.presence, cand.x, st);
            if (!st.valid || !st.stable)
                continue;
            const double g = dimensionlessGibbs(P, T, cand);
            if (isfinite(g) && g < bestG)
            {
                bestG = g;
                best = cand;
            }
        }
    }

    // preferStableSwReducedOverSingle_ (restricted.inc:703-780)
    NZ_HDN void preferStableSwReducedOverSingle(double P, double T, const double *z,
                                                                 Result<NC> &cand)
    {
        if (!sw() || popcount3(presenceFromFractions(cand.beta)) != 1)
            return;
        cand.presence = presenceFromFractions(cand.beta);
        StabilityResult<NC> single;
        stabilityTest(P, T, z, cand.presence, cand.x, single);
        const bool singleKnownUnstable = single.valid && !single.stable;
        Result<NC> reduced, trial;
        reduced.init();
        double reducedG = nzInf();
        const uint8_t pairs[3] = {OIL_BIT | GAS_BIT, OIL_BIT | WATER_BIT, GAS_BIT | WATER_BIT};
        for (int k = 0; k < 3; ++k)
        {
            flashRestricted(P, T, z, pairs[k], nullptr, trial);
            if (err)
                return;
            if (!trial.converged)
                continue;
            trial.presence = presenceFromFractions(trial.beta);
            if (trial.presence == 0)
                continue;
            StabilityResult<NC> st;
            stabilityTest(P, T, z, trial.presence, trial.x, st);
            if (!st.valid || !st.stable)
                continue;
            const double g = dimensionlessGibbs(P, T, trial);
            if (isfinite(g) && g < reducedG)
            {
                reducedG = g;
                reduced = trial;
            }
        }
        if (!reduced.converged)
        {
            if (singleKnownUnstable)
                cand.converged = false;
            return;
        }
        const double candG = dimensionlessGibbs(P, T, cand);
        const double scale = smax3(1.0, fabs(candG), fabs(reducedG));
        if (isfinite(reducedG) && (!isfinite(candG) || reducedG < candG - 1.0e-12 * scale))
        {
            cand = reduced;
            return;
        }
        if (singleKnownUnstable)
            cand.converged = false;
    }

    // numericalSwRoleResult_ (restricted.inc:514-541)
    NZ_HDN void numericalSwRoleResult(const Result<NC> &c, Result<NC> &n) const
    {
        n = c;
        if (!sw())
            return;
        for (int p = 0; p < 3; ++p)
        {
            n.beta[p] = 0.0;
            n.sat[p] = 0.0;
            n.Z[p] = 1.0;
            n.rho[p] = 0.0;
#pragma unroll
            for (int i = 0; i < NC; ++i)
                n.x[p][i] = 0.0;
        }
        for (int s = 0; s < 3; ++s)
        {
            const int phys = roles[s];
            n.beta[s] = c.beta[phys];
            n.sat[s] = c.sat[phys];
            n.Z[s] = c.Z[phys];
            n.rho[s] = c.rho[phys];
#pragma unroll
            for (int i = 0; i < NC; ++i)
                n.x[s][i] = c.x[phys][i];
        }
        n.presence = presenceFromFractions(n.beta);
        deriveReferenceK(n);
    }

    // One fixed role permutation of recovery 4: the nested flash under roles
    // swRolePermutation(k) (no permutation search, no continuation), whether
    // its answer is usable and its Gibbs energy under those roles.  An error
    // of the nested flash is this solver's error.
    NZ_HDN void permutedFlash(double P, double T, const double *z, int k, Result<NC> &permuted, bool &ok,
                              double &g)
    {
        int perm[3];
        swRolePermutation(k, perm);
        Solver<NC> cand = *this;
        cand.stabMemo = nullptr;   // stored tests were taken with the default roles
        cand.allocMemo = nullptr;
        cand.permMemo = nullptr;
        cand.roles[0] = perm[0];
        cand.roles[1] = perm[1];
        cand.roles[2] = perm[2];
        cand.permutationSearch = false;
        cand.continuation = false;
        cand.template flash<false>(P, T, z, permuted);
        ok = permuted.converged && cand.err == ERR_NONE;
        g = ok ? cand.dimensionlessGibbs(P, T, permuted) : 0.0;
        evals = cand.evals;
        if (cand.err)
            fail(cand.err);
    }

    // --------------------------------------------------------------- flash --
    // flash (three_phase_flash.hpp:83-227).  The nested solvers of the
    // role-permutation search and the pressure continuation run with both
    // recoveries disabled, exactly like the reference (core.inc:47-57).
    template <bool TopLevel>
    NZ_HDN void flash(double P, double T, const double *zIn, Result<NC> &out)
    {
        if (TopLevel && flashMemo)
        {
            bool hit = flashMemo->matches(P, T, zIn);
#ifdef __CUDA_ARCH__
            // warp-cooperative lanes take the stored answer together or not at all
            if (width > 1)
                hit = __all_sync(0xffffffffu, hit);
#endif
            if (hit)
            {
                out = flashMemo->r;
                if (flashMemo->err)
                    fail(flashMemo->err);
                return;
            }
        }
        out.init();
        if (!validatePT(P, T))
            return;
        double z[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            z[i] = zIn[i];
        normalize(z);
        if (err)
            return;
        double kg[NC], kw[NC];
        wilsonK(P, T, kg);
        initialWaterK(kw);

        Result<NC> seed;
        flashTwo(P, T, z, OIL, GAS, kg, seed);
        uint8_t active = presenceFromFractions(seed.beta);
        if (!seed.converged || active == 0)
        {
            active = chooseSinglePhase(P, T, z);
            singlePhaseResult(P, T, z, active, seed);
        }
        if (err)
            return;
        Result<NC> &selected = out;
        equilibrateActiveSet(P, T, z, active, seed, true, selected);
        if (err)
            return;
        if (selected.converged)
        {
            canonicalizeFinal(P, T, selected, false);
            if (selected.converged && validatePhysical(P, T, z, selected))
            {
                Result<NC> preferred = selected;
                preferStableSwReducedOverSingle(P, T, z, preferred);
                if (preferred.converged)
                {
                    out = preferred;
                    return;
                }
            }
            selected.converged = false;
        }
        if (err)
            return;
        recover<TopLevel>(P, T, z, out);
    }

    // The fail-only recoveries of flash() (three_phase_flash.hpp:122-224), run
    // when the active-set path did not give an accepted result.  On entry out
    // holds that failed result (converged == false) and z is normalised; out is
    // replaced by the first recovery that succeeds.  `from` > 1 skips the
    // recoveries before it (they already ran and failed).
    template <bool TopLevel>
    NZ_HDN void recover(double P, double T, const double *z, Result<NC> &out, int from = 1)
    {
        double kg[NC], kw[NC];
        wilsonK(P, T, kg);
        initialWaterK(kw);
        // recovery 1: direct three-phase solve
        if (from <= 1)
        {
            Result<NC> full;
            flashThree(P, T, z, kg, kw, full);
            if (full.converged)
            {
                canonicalize(P, T, full);
                canonicalizeFinal(P, T, full, false);
                if (full.converged && validatePhysical(P, T, z, full))
                {
                    preferStableSwReducedOverSingle(P, T, z, full);
                    if (full.converged)
                    {
                        out = full;
                        return;
                    }
                }
            }
        }
        if (err)
            return;
        // recovery 2: stable reduced phase sets
        if (from <= 2)
        {
            Result<NC> reduced;
            stableReducedSetFallback(P, T, z, reduced);
            if (reduced.converged)
            {
                canonicalizeFinal(P, T, reduced, false);
                if (reduced.converged && validatePhysical(P, T, z, reduced))
                {
                    out = reduced;
                    return;
                }
            }
        }
        if (err)
            return;
        if (from <= 3 && sw())
        {
            // recovery 3 (SW only): exact-mass allocation basin search
            Result<NC> allocated;
            allocationFallback(P, T, z, allocated);
            if (err)
                return;
            if (allocated.converged)
            {
                canonicalizeFinal(P, T, allocated, false);
                if (allocated.converged && validatePhysical(P, T, z, allocated))
                {
                    preferStableSwReducedOverSingle(P, T, z, allocated);
                    if (allocated.converged)
                    {
                        out = allocated;
                        return;
                    }
                }
            }
        }
        if (TopLevel && sw() && permutationSearch && from <= 4)
        {
            // recovery 4 (SW only): the other fixed role permutations (three_phase_flash.hpp:174-205)
            if (stopAtPermutations)
            {
                reachedPermutations = true;
                return;
            }
            const bool replay = permMemo && roles[0] == OIL && roles[1] == GAS && roles[2] == WATER &&
                                permMemo->matches(P, T, salinity, z);
            Result<NC> bestPermuted, permuted;
            bestPermuted.init();
            double bestG = nzInf();
#pragma unroll 1
            for (int k = 0; k < 6; ++k)
            {
                int perm[3];
                swRolePermutation(k, perm);
                if (perm[0] == roles[0] && perm[1] == roles[1] && perm[2] == roles[2])
                    continue;
                bool ok;
                double g;
                if (replay)
                {
                    const PermOut<NC> &o = permMemo->perm[k];
                    if (o.err)
                    {
                        fail(o.err);
                        return;
                    }
                    ok = o.ok != 0;
                    g = o.gibbs;
                    permuted = o.r;
                }
                else
                {
                    permutedFlash(P, T, z, k, permuted, ok, g);
                    if (err)
                        return;
                }
                if (!ok)
                    continue;
                if (isfinite(g) && g < bestG)
                {
                    bestG = g;
                    bestPermuted = permuted;
                }
            }
            if (bestPermuted.converged)
            {
                preferStableSwReducedOverSingle(P, T, z, bestPermuted);
                if (bestPermuted.converged)
                {
                    out = bestPermuted;
                    return;
                }
            }
        }
        if (TopLevel && continuation)
        {
            Result<NC> continued;
            pressureContinuation(P, T, z, continued);
            acceptContinued(P, T, z, continued, out);
        }
    }

    // One anchor of pressureContinuationFallback_ (restricted.inc:554-627): the
    // anchor flash at P * ratio[a], then the log-pressure path to P seeded by it.
    // Returns CONT_NONE (anchor or path did not converge), CONT_SUCCESS (out
    // holds the continued result) or CONT_ERROR (err is set).  Anchors are
    // independent of one another, so they may run in any order or in parallel;
    // the fallback's answer is that of the first anchor that is not CONT_NONE.
    // Pressure ratio of anchor a (restricted.inc:554-627).
    NZ_HD static double continuationRatio(int a)
    {
        const double ratios[8] = {0.95, 1.05, 0.90, 1.10, 0.80, 1.25, 0.65, 1.50};
        return ratios[a];
    }

    NZ_HDN int continuationAnchor(double P, double T, const double *z, int a, Result<NC> &out)
    {
        const double anchorP = P * continuationRatio(a);
        if (!(anchorP > 0.0) || !isfinite(anchorP))
            return CONT_NONE;
        Result<NC> anchor;
        {
            Solver<NC> nested = *this;
            nested.permutationSearch = false;
            nested.continuation = false;
            nested.template flash<false>(anchorP, T, z, anchor);
            evals = nested.evals;
            if (nested.err)
            {
                fail(nested.err);
                return CONT_ERROR;
            }
        }
        return continuationPath(P, T, z, a, anchor, out);
    }

    // The log-pressure path of anchor a from its converged anchor flash
    // `anchor` (taken at P * continuationRatio(a)) to P.
    NZ_HDN int continuationPath(double P, double T, const double *z, int a, const Result<NC> &anchor,
                                Result<NC> &out)
    {
        const double anchorP = P * continuationRatio(a);
        Result<NC> current;
        if (!anchor.converged)
            return CONT_NONE;
        numericalSwRoleResult(anchor, out);
        if (!out.converged || out.presence == 0)
            return CONT_NONE;
        const double logTarget = log(P);
        const double logAnchor = log(anchorP);
        const double logSpan = fabs(logTarget - logAnchor);
        int steps = int(ceil(logSpan / 0.025));
        steps = steps < 1 ? 1 : (steps > 12 ? 12 : steps);
        int totalIterations = anchor.iterations;
#pragma unroll 1
        for (int s = 1; s <= steps; ++s)
        {
            const double fraction = double(s) / steps;
            const double stepP = exp(logAnchor + fraction * (logTarget - logAnchor));
            equilibrateActiveSet(stepP, T, z, out.presence, out, false, current);
            if (err)
                return CONT_ERROR;
            if (!current.converged)
                return CONT_NONE;
            totalIterations += current.iterations;
            out = current;
        }
        if (!out.converged)
            return CONT_NONE;
        out.iterations = totalIterations;
        return CONT_SUCCESS;
    }

    // ---------------------------------------------------------- polish --
    // Final ln-fugacity Newton polish of a converged multiphase result (no
    // reference counterpart: the reference stops at its 1e-9 ln K tolerance,
    // which leaves ln-fugacity differences up to ~1e-9).  Newton on ln K with
    // the flash's own residual (evalTwo / evalThree: Rachford-Rice inside) and
    // a forward-difference Jacobian, until the largest residual is below
    // `target` or `maxSteps` steps are done.  `r` is replaced only by a state
    // with the same phases, a smaller residual and values within `maxChange`
    // of r's; an error inside leaves `r` and `err` as they were.  Returns true
    // when `r` was replaced.
    NZ_HDN bool polish(double P, double T, const double *z, Result<NC> &r, double target, int maxSteps,
                       double maxChange = 1.0e-8)
    {
        if (!r.converged)
            return false;
        const int errBefore = err;
        err = ERR_NONE;
        bool replaced = false;
        Result<NC> q = r;
        const int count = popcount3(r.presence);
        if (count == 2)
            replaced = polishTwo(P, T, z, q, target, maxSteps);
        else if (count == 3)
            replaced = polishThree(P, T, z, q, target, maxSteps);
        err = errBefore;
        if (!replaced)
            return false;
        // A converged answer is within its own tolerance of the exact one; a
        // polish that moves a fraction or a mole fraction further than
        // maxChange (relative to max(1, |v|)) has found a different, badly
        // conditioned solution next to a phase boundary: keep the answer.
        double change = 0.0;
#pragma unroll
        for (int p = 0; p < 3; ++p)
        {
            if (!(r.presence & bitOf(p)))
                continue;
            change = smax(change, fabs(q.beta[p] - r.beta[p]) / smax(1.0, fabs(r.beta[p])));
#pragma unroll
            for (int i = 0; i < NC; ++i)
                change = smax(change, fabs(q.x[p][i] - r.x[p][i]) / smax(1.0, fabs(r.x[p][i])));
        }
        if (!(change <= maxChange))
            return false;
        r = q;
        return true;
    }

    // The answer's phases evaluate, in their slots' roles, to the
    // compressibilities the answer records: the polish works in those roles
    // (an answer of the SW role search that does not has other roles or roots).
    NZ_HD bool sameRoots(const Result<NC> &r, const Result<NC> &e) const
    {
#pragma unroll
        for (int p = 0; p < 3; ++p)
            if ((r.presence & bitOf(p)) && !(fabs(e.Z[p] - r.Z[p]) <= 1.0e-6 * smax(1.0, fabs(r.Z[p]))))
                return false;
        return true;
    }

    NZ_HDN bool polishTwo(double P, double T, const double *z, Result<NC> &r, double target, int maxSteps)
    {
        int first, second;
        activePair(r.presence, first, second);
        double logK[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i)
            logK[i] = log(smax(r.x[second][i], O().floor) / smax(r.x[first][i], O().floor));
        TwoPhaseLogKState<NC> base, probe;
        evalTwo(P, T, z, first, second, logK, r.beta[second], base);
        if (!base.valid || err || !sameRoots(r, base.result))
            return false;
        const double start = base.norm;
        bool moved = false;
#pragma unroll 1
        for (int step = 0; step < maxSteps && base.norm > target; ++step)
        {
            double J[NC][NC];
            bool ok = true;
#pragma unroll 1
            for (int col = 0; col < NC && ok; ++col)
            {
                double pert[NC];
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    pert[i] = logK[i];
                // forward difference, backward where the forward probe leaves the
                // admissible fractions (a small phase close to zero)
                double h = O().fdStep * smax(1.0, fabs(logK[col]));
                pert[col] = logK[col] + h;
                evalTwo(P, T, z, first, second, pert, base.result.beta[second], probe);
                if (!probe.valid || err)
                {
                    err = ERR_NONE;
                    h = -h;
                    pert[col] = logK[col] + h;
                    evalTwo(P, T, z, first, second, pert, base.result.beta[second], probe);
                }
                ok = probe.valid && !err;
                if (ok)
#pragma unroll
                    for (int row = 0; row < NC; ++row)
                        J[row][col] = (probe.residual[row] - base.residual[row]) / h;
            }
            double rhs[NC], delta[NC];
#pragma unroll
            for (int i = 0; i < NC; ++i)
                rhs[i] = -base.residual[i];
            if (!ok || !solveDense<NC>(J, rhs, delta))
                break;
            bool accepted = false;
            double damping = 1.0;
#pragma unroll 1
            for (int ls = 0; ls < 8 && !accepted; ++ls, damping *= 0.5)
            {
                double trial[NC];
#pragma unroll
                for (int i = 0; i < NC; ++i)
                    trial[i] = logK[i] + damping * delta[i];
                evalTwo(P, T, z, first, second, trial, base.result.beta[second], probe);
                if (probe.valid && !err && probe.norm < base.norm)
                {
#pragma unroll
                    for (int i = 0; i < NC; ++i)
                        logK[i] = trial[i];
                    base = probe;
                    accepted = moved = true;
                }
            }
            if (!accepted)
                break;
        }
        if (!moved || !(base.norm < start))
            return false;
        Result<NC> q = r;
        q.beta[0] = q.beta[1] = q.beta[2] = 0.0;
        q.beta[first] = base.result.beta[first];
        q.beta[second] = base.result.beta[second];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            q.x[first][i] = base.result.x[first][i];
            q.x[second][i] = base.result.x[second][i];
        }
        q.Z[first] = base.result.Z[first];
        q.Z[second] = base.result.Z[second];
        if (presenceFromFractions(q.beta) != r.presence)
            return false;
        // the K-values stay the answer's (a move of at most maxChange leaves
        // them consistent; SW answers do not define them from x alone)
        updateSaturations(P, T, q);
        if (err)
            return false;
        r = q;
        return true;
    }

    NZ_HDN bool polishThree(double P, double T, const double *z, Result<NC> &r, double target, int maxSteps)
    {
        constexpr int M = 2 * NC;
        double logK[M];
#pragma unroll
        for (int i = 0; i < NC; ++i)
        {
            const double xo = smax(r.x[0][i], O().floor);
            logK[i] = log(smax(r.x[1][i], O().floor) / xo);
            logK[NC + i] = log(smax(r.x[2][i], O().floor) / xo);
        }
        ThreePhaseLogKState<NC> base, probe;
        evalThree(P, T, z, logK, r.beta[1], r.beta[2], base);
        if (!base.valid || err || !sameRoots(r, base.result))
            return false;
        const double start = base.norm;
        bool moved = false;
#pragma unroll 1
        for (int step = 0; step < maxSteps && base.norm > target; ++step)
        {
            double J[M][M];
            bool ok = true;
#pragma unroll 1
            for (int col = 0; col < M && ok; ++col)
            {
                double pert[M];
#pragma unroll
                for (int i = 0; i < M; ++i)
                    pert[i] = logK[i];
                double h = O().fdStep * smax(1.0, fabs(logK[col]));
                pert[col] = logK[col] + h;
                evalThree(P, T, z, pert, base.result.beta[1], base.result.beta[2], probe);
                if (!probe.valid || err)
                {
                    err = ERR_NONE;
                    h = -h;
                    pert[col] = logK[col] + h;
                    evalThree(P, T, z, pert, base.result.beta[1], base.result.beta[2], probe);
                }
                ok = probe.valid && !err;
                if (ok)
#pragma unroll
                    for (int row = 0; row < M; ++row)
                        J[row][col] = (probe.residual[row] - base.residual[row]) / h;
            }
            double rhs[M], delta[M];
#pragma unroll
            for (int i = 0; i < M; ++i)
                rhs[i] = -base.residual[i];
            if (!ok || !solveDense<M>(J, rhs, delta))
                break;
            bool accepted = false;
            double damping = 1.0;
#pragma unroll 1
            for (int ls = 0; ls < 8 && !accepted; ++ls, damping *= 0.5)
            {
                double trial[M];
#pragma unroll
                for (int i = 0; i < M; ++i)
                    trial[i] = logK[i] + damping * delta[i];
                evalThree(P, T, z, trial, base.result.beta[1], base.result.beta[2], probe);
                if (probe.valid && !err && probe.norm < base.norm)
                {
#pragma unroll
                    for (int i = 0; i < M; ++i)
                        logK[i] = trial[i];
                    base = probe;
                    accepted = moved = true;
                }
            }
            if (!accepted)
                break;
        }
        if (!moved || !(base.norm < start))
            return false;
        Result<NC> q = r;
#pragma unroll
        for (int p = 0; p < 3; ++p)
        {
            q.beta[p] = base.result.beta[p];
            q.Z[p] = base.result.Z[p];
#pragma unroll
            for (int i = 0; i < NC; ++i)
                q.x[p][i] = base.result.x[p][i];
        }
        if (presenceFromFractions(q.beta) != r.presence)
            return false;
        // the K-values stay the answer's (a move of at most maxChange leaves
        // them consistent; SW answers do not define them from x alone)
        updateSaturations(P, T, q);
        if (err)
            return false;
        r = q;
        return true;
    }

    // pressureContinuationFallback_ (restricted.inc:554-627): anchors in order.
    NZ_HDN void pressureContinuation(double P, double T, const double *z, Result<NC> &out)
    {
        out.init();
        if (!(P > 0.0))
            return;
        Result<NC> continued;
#pragma unroll 1
        for (int a = 0; a < 8; ++a)
        {
            const int outcome = continuationAnchor(P, T, z, a, continued);
            if (outcome == CONT_ERROR)
                return;
            if (outcome == CONT_SUCCESS)
            {
                out = continued;
                return;
            }
        }
    }

    // What flash() does with a continued result (three_phase_flash.hpp:206-224):
    // out is replaced only when the result survives the final checks.
    NZ_HDN void acceptContinued(double P, double T, const double *z, Result<NC> &continued, Result<NC> &out)
    {
        if (!continued.converged)
            return;
        canonicalizeFinal(P, T, continued, false);
        if (continued.converged && validatePhysical(P, T, z, continued))
        {
            preferStableSwReducedOverSingle(P, T, z, continued);
            if (continued.converged)
                out = continued;
        }
    }
};

} // namespace nz
