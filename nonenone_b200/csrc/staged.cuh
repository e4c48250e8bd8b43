// staged.cuh -- the batched flash split at its stability tests.
//
// The reference's flash (three_phase_flash.hpp:83-227) spends most of its
// EOS evaluations in the multi-seed TPD stability tests that the active-set
// loop (three_phase_flash_allocation.inc:707-858) runs after every
// equilibrium of a reduced phase set.  One thread per point running the whole
// pipeline leaves ~3 of 32 lanes active.  Here the active-set loop of every
// point is a resumable state machine:
//
//   driver kernel   runs the reference's control flow for one point until it
//                   needs a stability test, writes the test's reference-phase
//                   data and one task per missing phase, and suspends;
//   trial kernel    runs every (task, seed) TPD trial as its own lane, one EOS
//                   evaluation per loop step, lanes refilled from a global
//                   queue (stability.inc:225-355 restated as a step machine);
//   driver resume   combines the trials in seed order exactly like
//                   stabilityTest (three_phase_flash.hpp:393-487) and
//                   continues the loop.
//
// Only the main path is staged.  A point whose main path does not end in a
// validated result (the reference then tries its fail-only recoveries) is
// queued for the full per-thread solver, which recomputes it from scratch.
#pragma once

#include "flash.cuh"

namespace nz
{

constexpr uint8_t STAGE_DONE = 0;
constexpr uint8_t STAGE_NEED_STABILITY = 1;
constexpr uint8_t STAGE_NEED_FULL = 2;
constexpr uint8_t STAGE_NEED_THREE = 3;   // suspended at a three-phase solve (flashThree_)

// Per-point state kept in HBM between driver launches.
template <int NC>
struct DriverState
{
    double P, T, sal;
    double z[NC];
    Result<NC> seed;
    Result<NC> lastPhysical;
    Result<NC> current;
    // pending stability request (three_phase_flash.hpp:300-393)
    double refX[NC];
    double logRef[NC];
    double sx[3][NC];
    StabilityResult<NC> sr;   // the combined result of the last stability test
    unsigned long long evals;
    int err;
    uint8_t active;
    uint8_t outer;
    uint8_t useConvergedSeed;
    uint8_t stage;
    uint8_t tested;
    uint8_t mainFailed;   // the active-set path ended without an accepted result and without an error
    uint8_t recoverFrom;  // for the warp recovery kernel: 0 = flash() from scratch, else the first recovery to run
    uint8_t r2Cand;       // recovery 2: the candidate pair under test / next to try
    double r2BestG;       // recovery 2: Gibbs energy of the best certified candidate (in `seed`)
    double threeKg[NC];   // starting K of the pending three-phase solve
    double threeKw[NC];
    int allocSlot;        // SW allocation search precomputed in this memo slot (-1: none)
};

template <int NC>
struct TrialOut
{
    double sum;
    double x[NC];
    int valid;
    int trivial;
};

// Queues of one staged flash call (device memory, owned by the context).
struct StagedQueues
{
    unsigned long long *tasks[2];   // (point << 2) | candidate phase
    int *pending[2];                // points waiting for their trials
    int *full;                      // points for the full solver
    int *counters;                  // [rounds][4]: tasks, pending, trial cursor, spare; + full at the end
};

constexpr int kMaxRounds = 9;   // one stability test per active-set outer pass (<= 8) + 1

template <int NC>
NZ_BOTH int seedCount(const FluidDev &F)
{
    return NC + 6 + ((F.water >= 0 && NC > 1) ? 1 : 0);
}

// ---------------------------------------------------------------- driver --
template <int NC>
struct Driver
{
    Solver<NC> s;
    DriverState<NC> *st;

    // stabilityTest up to the trials (three_phase_flash.hpp:300-393).
    // Returns false when the test resolves without trials (SW certification
    // failure -> invalid); `res` then holds the result.
    NZ_HD bool prepareStability(double P, double T, const double *zIn, uint8_t active,
                                const double (&activeX)[3][NC], StabilityResult<NC> &res)
    {
        res.stable = true;
        res.valid = true;
        res.tested = active;
        for (int p = 0; p < 3; ++p)
        {
            res.unstable[p] = false;
            res.trialSum[p] = 1.0;
            for (int i = 0; i < NC; ++i)
                res.incipient[p][i] = 0.0;
        }
        if (!s.validatePT(P, T) || active == 0)
        {
            s.fail(ERR_BAD_INPUT);
            return false;
        }
        double z[NC];
        for (int i = 0; i < NC; ++i)
            z[i] = zIn[i];
        s.normalize(z);
        const int ref = firstActive(active);
        for (int p = 0; p < 3; ++p)
            for (int i = 0; i < NC; ++i)
                st->sx[p][i] = activeX[p][i];
        if (s.sw() && popcount3(active) == 1)
            for (int i = 0; i < NC; ++i)
                st->sx[ref][i] = z[i];
        for (int p = 0; p < 3; ++p)
            if (active & bitOf(p))
                s.normalize(st->sx[p]);
        if (s.sw() && popcount3(active) > 1)
        {
            double phiR[NC], phiP[NC];
            s.phase(ref, P, T, st->sx[ref], phiR);
            double mismatch = 0.0;
            for (int p = 0; p < 3; ++p)
            {
                if (!(active & bitOf(p)) || p == ref)
                    continue;
                s.phase(p, P, T, st->sx[p], phiP);
                for (int i = 0; i < NC; ++i)
                {
                    const double xr = st->sx[ref][i], xp = st->sx[p][i];
                    if (xr <= 10.0 * s.O().floor || xp <= 10.0 * s.O().floor)
                        continue;
                    mismatch = smax(mismatch, fabs(log(smax(xr * phiR[i], 1.0e-300) /
                                                       smax(xp * phiP[i], 1.0e-300))));
                }
            }
            if (mismatch > smax(10.0 * s.O().fugacityTol, 10.0 * s.O().stabilityTol))
            {
                Result<NC> certified;
                s.flashRestrictedImpl(P, T, z, active, &st->sx, certified);
                if (!certified.converged || certified.presence != active)
                {
                    res.valid = false;
                    res.stable = false;
                    return false;
                }
                for (int p = 0; p < 3; ++p)
                    for (int i = 0; i < NC; ++i)
                        st->sx[p][i] = certified.x[p][i];
            }
        }
        for (int i = 0; i < NC; ++i)
            st->refX[i] = st->sx[ref][i];
        s.normalize(st->refX);
        double phiRef[NC];
        s.phase(ref, P, T, st->refX, phiRef);
        for (int i = 0; i < NC; ++i)
            st->logRef[i] = log(smax(st->refX[i], s.O().floor)) + log(smax(phiRef[i], 1.0e-300));
        st->tested = active;
        return true;
    }

    // The trial-combination half of stabilityTest (three_phase_flash.hpp:393-487).
    NZ_HD void combineStability(const TrialOut<NC> *trials, int nseeds, StabilityResult<NC> &res)
    {
        const uint8_t active = st->tested;
        res.stable = true;
        res.valid = true;
        res.tested = active;
        for (int p = 0; p < 3; ++p)
        {
            res.unstable[p] = false;
            res.trialSum[p] = 1.0;
            for (int i = 0; i < NC; ++i)
                res.incipient[p][i] = 0.0;
        }
        const double coincTol = smax(10.0 * s.O().coincidentTol, 1.0e-7);
        for (int cand = 0; cand < 3; ++cand)
        {
            if (active & bitOf(cand))
                continue;
            int best = -1;
            for (int k = 0; k < nseeds; ++k)
            {
                const TrialOut<NC> &t = trials[cand * nseeds + k];
                if (t.valid && (best < 0 || t.sum > trials[cand * nseeds + best].sum))
                    best = k;
            }
            if (best < 0)
            {
                res.valid = false;
                res.stable = false;
                continue;
            }
            const TrialOut<NC> &b = trials[cand * nseeds + best];
            res.trialSum[cand] = b.sum;
            for (int i = 0; i < NC; ++i)
                res.incipient[cand][i] = b.x[i];
            bool coincides = false;
            for (int p = 0; p < 3; ++p)
            {
                if (!(active & bitOf(p)))
                    continue;
                double maxDiff = 0.0;
                for (int i = 0; i < NC; ++i)
                    maxDiff = smax(maxDiff, fabs(b.x[i] - st->sx[p][i]));
                if (maxDiff <= coincTol)
                {
                    coincides = true;
                    break;
                }
            }
            const bool unstable = !b.trivial && !coincides && b.sum > 1.0 + s.O().stabilityTol;
            res.unstable[cand] = unstable;
            res.stable = res.stable && !unstable;
        }
        // a trial that stopped on an EOS error aborts the test, as in the
        // sequential loop (the lowest-index error wins)
        for (int cand = 0; cand < 3; ++cand)
        {
            if (active & bitOf(cand))
                continue;
            for (int k = 0; k < nseeds; ++k)
                if (trials[cand * nseeds + k].valid < 0)
                {
                    s.fail(-trials[cand * nseeds + k].valid);
                    return;
                }
        }
    }

    // ----------------------------------------------- fail-only recoveries --
    // Recovery 1 of flash() (three_phase_flash.hpp:122-141) after a failed
    // active-set path.  True when it decides the point: st->current is then
    // the answer, or s.err is set.
    NZ_HD bool recoveryOne()
    {
        double kg[NC], kw[NC];
        s.wilsonK(st->P, st->T, kg);
        s.initialWaterK(kw);
        Result<NC> full;
        s.flashThree(st->P, st->T, st->z, kg, kw, full);
        return recoveryOneAccept(full);
    }

    // The starting K of recovery 1's three-phase solve (Wilson, initial water).
    NZ_HD void recoveryOneStart()
    {
        s.wilsonK(st->P, st->T, st->threeKg);
        s.initialWaterK(st->threeKw);
    }

    // What flash() does with recovery 1's three-phase result `full`.
    NZ_HD bool recoveryOneAccept(Result<NC> &full)
    {
        const double P = st->P, T = st->T;
        if (full.converged)
        {
            s.canonicalize(P, T, full);
            s.canonicalizeFinal(P, T, full, false);
            if (full.converged && s.validatePhysical(P, T, st->z, full))
            {
                s.preferStableSwReducedOverSingle(P, T, st->z, full);
                if (full.converged)
                {
                    st->current = full;
                    return true;
                }
            }
        }
        return s.err != ERR_NONE;
    }

    // stableReducedSetFallback_ (restricted.inc:655-693) as a resumable loop
    // over the candidate pairs O+G, O+W, G+W.  Advances from pair st->r2Cand;
    // returns STAGE_NEED_STABILITY with the stability request of that pair's
    // candidate (held in st->lastPhysical) prepared, or STAGE_DONE when the
    // pairs are exhausted or s.err is set.  The best certified candidate is
    // kept in st->seed with its Gibbs energy in st->r2BestG.
    NZ_HD uint8_t reducedAdvance()
    {
        const uint8_t pairs[3] = {OIL_BIT | GAS_BIT, OIL_BIT | WATER_BIT, GAS_BIT | WATER_BIT};
        const double P = st->P, T = st->T;
        Result<NC> &cand = st->lastPhysical;
        while (st->r2Cand < 3)
        {
            s.flashRestrictedRecovery(P, T, st->z, pairs[st->r2Cand], cand);
            if (s.err)
                return STAGE_DONE;
            if (cand.converged)
            {
                cand.presence = s.presenceFromFractions(cand.beta);
                if (cand.presence != 0)
                {
                    StabilityResult<NC> direct;
                    if (prepareStability(P, T, st->z, cand.presence, cand.x, direct))
                        return STAGE_NEED_STABILITY;
                    if (s.err)
                        return STAGE_DONE;
                    // resolved without trials: not valid, the candidate is rejected
                }
            }
            ++st->r2Cand;
        }
        return STAGE_DONE;
    }

    // The trials of the pair under test are in: certify and rank its candidate.
    NZ_HD void reducedCombine(const TrialOut<NC> *trials, int nseeds)
    {
        StabilityResult<NC> sr;
        combineStability(trials, nseeds, sr);
        if (s.err)
            return;
        if (sr.valid && sr.stable)
        {
            const double g = s.dimensionlessGibbs(st->P, st->T, st->lastPhysical);
            if (isfinite(g) && g < st->r2BestG)
            {
                st->r2BestG = g;
                st->seed = st->lastPhysical;
            }
        }
        ++st->r2Cand;
    }

    // flash()'s acceptance of the recovery-2 answer (three_phase_flash.hpp:143-157).
    NZ_HD bool reducedFinish()
    {
        Result<NC> &reduced = st->seed;
        if (!reduced.converged)
            return false;
        s.canonicalizeFinal(st->P, st->T, reduced, false);
        if (reduced.converged && s.validatePhysical(st->P, st->T, st->z, reduced))
        {
            st->current = reduced;
            return true;
        }
        return false;
    }

    // equilibrateActiveSet_ as a resumable loop (allocation.inc:707-858).
    // Returns STAGE_NEED_STABILITY when it suspended for a stability test,
    // otherwise it has stored the loop's result in st->current.
    NZ_HD uint8_t activeSetLoop(bool resumed, const StabilityResult<NC> *resumedSt, bool afterThree = false)
    {
        const double P = st->P, T = st->T;
        const double *z = st->z;
        Result<NC> &seed = st->seed;
        Result<NC> &current = st->current;
        Result<NC> &lastPhysical = st->lastPhysical;
        uint8_t active = st->active;
        bool useConvergedSeed = st->useConvergedSeed != 0;
        int outer = st->outer;
        bool afterStability = resumed;
        while (outer < 8)
        {
            if (s.err)
                return STAGE_NEED_FULL;
            if (afterStability)
            {
                afterStability = false;
                const StabilityResult<NC> &sr = *resumedSt;
                if (!sr.valid)
                {
                    current.converged = false;
                    s.canonicalize(P, T, current);
                    return STAGE_DONE;
                }
                if (sr.stable)
                {
                    s.canonicalize(P, T, current);
                    return STAGE_DONE;
                }
                bool added = false;
                for (int p = 0; p < 3; ++p)
                {
                    if (!(active & bitOf(p)) && sr.unstable[p])
                    {
                        active |= uint8_t(bitOf(p));
                        for (int i = 0; i < NC; ++i)
                            seed.x[p][i] = sr.incipient[p][i];
                        added = true;
                    }
                }
                if (!added)
                {
                    current.converged = false;
                    s.canonicalize(P, T, current);
                    return STAGE_DONE;
                }
                s.deriveReferenceK(seed);
                seed.presence = active;
                useConvergedSeed = false;
                ++outer;
                continue;
            }
            if (afterThree)
            {
                // the three-phase solve this pass suspended at has written current
                afterThree = false;
                if (!current.converged)
                {
                    lastPhysical.converged = false;
                    s.canonicalize(P, T, lastPhysical);
                    current = lastPhysical;
                    return STAGE_DONE;
                }
            }
            else if (useConvergedSeed)
            {
                current = seed;
                useConvergedSeed = false;
            }
            else if (popcount3(active) == 1)
            {
                s.singlePhaseResult(P, T, z, active, current);
            }
            else if (popcount3(active) == 2)
            {
                int first, second;
                activePair(active, first, second);
                double K[NC];
                s.pairInitialK(first, second, P, T, z, K);
                if (seed.converged && seed.presence == active)
                    for (int i = 0; i < NC; ++i)
                        K[i] = sclamp(seed.x[second][i] / smax(seed.x[first][i], s.O().floor), 1.0e-100, 1.0e100);
                s.flashTwo(P, T, z, first, second, K, current);
                if (!current.converged)
                    s.singlePhaseResult(P, T, z, s.chooseSinglePhase(P, T, z), current);
            }
            else
            {
                double kg[NC], kw[NC];
                bool kgValid = true, kwValid = true;
                for (int i = 0; i < NC; ++i)
                {
                    kg[i] = seed.Kg[i];
                    kw[i] = seed.Kw[i];
                    kgValid = kgValid && kg[i] > 0.0;
                    kwValid = kwValid && kw[i] > 0.0;
                }
                if (!kgValid) s.wilsonK(P, T, kg);
                if (!kwValid) s.initialWaterK(kw);
                // flashThree runs on the three-phase kernel; the loop resumes above
                for (int i = 0; i < NC; ++i)
                {
                    st->threeKg[i] = kg[i];
                    st->threeKw[i] = kw[i];
                }
                st->active = active;
                st->outer = uint8_t(outer);
                st->useConvergedSeed = useConvergedSeed;
                return STAGE_NEED_THREE;
            }
            uint8_t fractionPresence = s.presenceFromFractions(current.beta);
            if (fractionPresence == 0)
                fractionPresence = s.chooseSinglePhase(P, T, z);
            if (fractionPresence != active)
            {
                active = fractionPresence;
                seed = current;
                s.canonicalize(P, T, seed);
                lastPhysical = seed;
                useConvergedSeed = seed.converged && seed.presence == active && !s.sw();
                ++outer;
                continue;
            }
            s.canonicalize(P, T, current);
            lastPhysical = current;
            if (popcount3(active) == 3)
            {
                s.canonicalize(P, T, current);
                return STAGE_DONE;
            }
            StabilityResult<NC> direct;
            if (!prepareStability(P, T, z, active, current.x, direct))
            {
                if (s.err)
                    return STAGE_NEED_FULL;
                // resolved without trials (invalid) -> same handling as after the test
                current.converged = false;
                s.canonicalize(P, T, current);
                return STAGE_DONE;
            }
            st->active = active;
            st->outer = uint8_t(outer);
            st->useConvergedSeed = useConvergedSeed;
            return STAGE_NEED_STABILITY;
        }
        s.canonicalize(P, T, seed);
        current = seed;
        return STAGE_DONE;
    }

    // flash() after the active-set loop: final canonicalisation, validation
    // and (SW) the reduced-set preference (three_phase_flash.hpp:106-120).
    // Returns STAGE_DONE with st->current the answer, or STAGE_NEED_FULL.
    NZ_HD uint8_t finish()
    {
        Result<NC> &selected = st->current;
        if (s.err)
            return STAGE_NEED_FULL;
        if (selected.converged)
        {
            s.canonicalizeFinal(st->P, st->T, selected, false);
            if (selected.converged && s.validatePhysical(st->P, st->T, st->z, selected))
            {
                s.preferStableSwReducedOverSingle(st->P, st->T, st->z, selected);
                if (selected.converged && !s.err)
                    return STAGE_DONE;
            }
        }
        // flash() marks the failed result and goes on to its recoveries
        selected.converged = false;
        st->mainFailed = s.err == ERR_NONE;
        return STAGE_NEED_FULL;
    }

    // flash() up to the active-set loop (three_phase_flash.hpp:87-104).
    NZ_HD uint8_t start(double P, double T, const double *zIn)
    {
        st->P = P;
        st->T = T;
        st->outer = 0;
        st->mainFailed = 0;
        st->current.init();
        if (!s.validatePT(P, T))
            return STAGE_NEED_FULL;
        for (int i = 0; i < NC; ++i)
            st->z[i] = zIn[i];
        s.normalize(st->z);
        if (s.err)
            return STAGE_NEED_FULL;
        double kg[NC];
        s.wilsonK(P, T, kg);
        Result<NC> &seed = st->seed;
        s.flashTwo(P, T, st->z, OIL, GAS, kg, seed);
        uint8_t active = s.presenceFromFractions(seed.beta);
        if (!seed.converged || active == 0)
        {
            active = s.chooseSinglePhase(P, T, st->z);
            s.singlePhaseResult(P, T, st->z, active, seed);
        }
        if (s.err)
            return STAGE_NEED_FULL;
        // equilibrateActiveSet_ prologue (allocation.inc:716-732)
        if (active == 0)
            active = s.chooseSinglePhase(P, T, st->z);
        s.canonicalize(P, T, seed);
        if (seed.presence != active)
            active = seed.presence;
        st->lastPhysical = seed;
        st->useConvergedSeed = seed.converged && seed.presence == active && !s.sw();
        st->active = active;
        return STAGE_DONE;
    }
};

// ----------------------------------------------------- trial step machine --
// One lane = one TPD trial of stabilityTrial_ (stability.inc:225-355), driven
// one EOS evaluation per step so every lane of a warp executes the EOS code
// together whatever phase of the trial it is in.
constexpr double kMixedSsiHandover = 1.0e-5;   // mixed form: FP32 residual below which FP64 SSI takes over
constexpr int TM_SSI = 0;        // leading SSI steps
constexpr int TM_NEWTON = 1;     // Newton base evaluation
constexpr int TM_FD = 2;         // finite-difference column evaluation
constexpr int TM_LINE = 3;       // line-search evaluation
constexpr int TM_TAIL = 4;       // remaining SSI budget

template <int NC>
struct TrialLane
{
    int mode;
    int it;            // iterations done in the current mode
    int newtonIt;
    int col;           // FD column / line-search step
    int candidate;
    bool fp64Ssi;      // mixed form: the leading SSI steps have gone over to FP64
    double P, T;
    double logW[NC];
    double logRef[NC];
    double ref[NC];
    double probe[NC];  // logW being evaluated (FD / line search)
    double step[NC];
    double baseRes[NC];
    double baseNorm;
    double J[NC][NC];
    double delta[NC];
    double damping;
};

// Start a trial: the seed's ln W (stability.inc:233-242).
template <int NC>
NZ_HD void trialInit(Solver<NC> &s, TrialLane<NC> &L, const double *seedIn)
{
    double seed[NC];
    for (int i = 0; i < NC; ++i)
        seed[i] = seedIn[i];
    s.normalize(seed);
    for (int i = 0; i < NC; ++i)
        L.logW[i] = log(smax(seed[i], s.O().floor));
    L.it = 0;
    L.newtonIt = 0;
    L.fp64Ssi = false;
    const int ssiSteps = imin(s.O().maxStability, imax(s.O().stabilitySsi, 0));
    L.mode = ssiSteps > 0 ? TM_SSI : (s.O().stabilityNewton > 0 ? TM_NEWTON : TM_TAIL);
}

// The mixed form's FP32 phase of a trial (run ahead of the FP64 steps, in its
// own kernel): leading SSI steps with FP32 mixing and ln phi (FP64 root),
// which never end a trial, until the FP32 residual is below
// kMixedSsiHandover, the leading budget is spent, or an FP32 evaluation
// fails; every later step is FP64.  Returns -1 when the trial ended invalid
// (an empty trailing budget), else 0 with L ready for the FP64 steps.
template <int NC>
NZ_HD bool trialEnterTail(Solver<NC> &s, TrialLane<NC> &L);

template <int NC>
NZ_HD int trialMixedPhase(Solver<NC> &s, TrialLane<NC> &L)
{
    const FlashOpts &O = s.O();
    const int ssiSteps = imin(O.maxStability, imax(O.stabilitySsi, 0));
    StabilityResidual<NC> r;
    while (L.mode == TM_SSI && !L.fp64Ssi)
    {
        if (!s.stabilityResidualMixed(L.candidate, L.P, L.T, L.logRef, L.logW, r))
            break;
        for (int i = 0; i < NC; ++i)
            L.logW[i] = L.logRef[i] - r.lnphi[i];
        ++L.it;
        if (L.it >= ssiSteps)
        {
            if (O.stabilityNewton > 0)
            {
                L.mode = TM_NEWTON;
                L.it = 0;
            }
            else if (!trialEnterTail(s, L))
                return -1;
        }
        else if (r.norm < kMixedSsiHandover)
            L.fp64Ssi = true;
    }
    L.fp64Ssi = true;
    return 0;
}

// Enter the trailing SSI budget; false when it is empty (trial invalid).
template <int NC>
NZ_HD bool trialEnterTail(Solver<NC> &s, TrialLane<NC> &L)
{
    const int ssiSteps = imin(s.O().maxStability, imax(s.O().stabilitySsi, 0));
    L.mode = TM_TAIL;
    L.it = 0;
    return imax(0, s.O().maxStability - ssiSteps) > 0;
}

template <int NC>
NZ_HD void trialSetProbeFd(Solver<NC> &s, TrialLane<NC> &L)
{
    for (int i = 0; i < NC; ++i)
        L.probe[i] = L.logW[i];
    L.step[L.col] = s.O().fdStep * smax(1.0, fabs(L.logW[L.col]));
    L.probe[L.col] += L.step[L.col];
}

// One EOS evaluation of the trial.  Returns 0 while running, 1 when the
// trial ended with a converged stationary point (written to `out`), -1 when
// it ended invalid.
template <int NC>
NZ_HD int trialStep(Solver<NC> &s, TrialLane<NC> &L, TrialOut<NC> &out)
{
    StabilityResidual<NC> r;
    const bool probing = L.mode == TM_FD || L.mode == TM_LINE;
    const FlashOpts &O = s.O();
    const int ssiSteps = imin(O.maxStability, imax(O.stabilitySsi, 0));
    s.stabilityResidual(L.candidate, L.P, L.T, L.logRef, probing ? L.probe : L.logW, r);
    switch (L.mode)
    {
    case TM_SSI:
    case TM_TAIL:
        if (!r.valid)
            return -1;
        if (r.norm < O.stabilityTol)
            break;   // converged
        for (int i = 0; i < NC; ++i)
            L.logW[i] = L.logRef[i] - log(smax(r.phi[i], 1.0e-300));
        ++L.it;
        if (L.mode == TM_SSI && L.it >= ssiSteps)
        {
            if (O.stabilityNewton > 0)
            {
                L.mode = TM_NEWTON;
                L.it = 0;
            }
            else if (!trialEnterTail(s, L))
                return -1;
        }
        else if (L.mode == TM_TAIL && L.it >= imax(0, O.maxStability - ssiSteps))
            return -1;
        return 0;
    case TM_NEWTON:
        if (!r.valid)
            return -1;
        if (r.norm < O.stabilityTol)
            break;
        for (int i = 0; i < NC; ++i)
            L.baseRes[i] = r.residual[i];
        L.baseNorm = r.norm;
        L.col = 0;
        L.mode = TM_FD;
        trialSetProbeFd(s, L);
        return 0;
    case TM_FD:
        if (!r.valid)
            return -1;
        for (int row = 0; row < NC; ++row)
            L.J[row][L.col] = (r.residual[row] - L.baseRes[row]) / L.step[L.col];
        if (++L.col < NC)
        {
            trialSetProbeFd(s, L);
            return 0;
        }
        {
            double J[NC][NC], rhs[NC];
            for (int a = 0; a < NC; ++a)
            {
                rhs[a] = -L.baseRes[a];
                for (int b = 0; b < NC; ++b)
                    J[a][b] = L.J[a][b];
            }
            if (!solveDense<NC>(J, rhs, L.delta))
                return trialEnterTail(s, L) ? 0 : -1;
        }
        L.damping = 1.0;
        L.col = 0;
        for (int i = 0; i < NC; ++i)
            L.probe[i] = L.logW[i] + L.damping * L.delta[i];
        L.mode = TM_LINE;
        return 0;
    case TM_LINE:
        if (r.valid && r.norm < L.baseNorm)
        {
            for (int i = 0; i < NC; ++i)
                L.logW[i] = L.probe[i];
            if (++L.newtonIt >= O.stabilityNewton)
                return trialEnterTail(s, L) ? 0 : -1;
            // The next Newton base evaluation is at this same ln W: reuse it
            // (the reference evaluates it again; the values are identical).
            if (r.norm < O.stabilityTol)
                break;
            for (int i = 0; i < NC; ++i)
                L.baseRes[i] = r.residual[i];
            L.baseNorm = r.norm;
            L.col = 0;
            L.mode = TM_FD;
            trialSetProbeFd(s, L);
            return 0;
        }
        L.damping *= 0.5;
        if (++L.col >= 16)
            return trialEnterTail(s, L) ? 0 : -1;
        for (int i = 0; i < NC; ++i)
            L.probe[i] = L.logW[i] + L.damping * L.delta[i];
        return 0;
    }
    // converged at the evaluated point: finalizeStabilityTrial_
    Trial<NC> t;
    s.finalizeTrial(r, L.ref, t);
    out.valid = 1;
    out.trivial = t.trivial;
    out.sum = t.sum;
    for (int i = 0; i < NC; ++i)
        out.x[i] = t.x[i];
    return 1;
}

// ---------------------------------------------------------- three-phase --
// flashThree_ (nonlinear.inc:279-513) as a step machine: every step is one
// threeSsiStep or one evalThree (one robust RR3 solve and three phase
// evaluations), so the lanes of a warp stay in step while each runs its own
// solve.  The steps and their order are those of Solver::flashThree.
constexpr int TH_SSI = 0;    // leading SSI steps
constexpr int TH_BASE = 1;   // Newton base evaluation
constexpr int TH_FD = 2;     // finite-difference column (forward, then backward if invalid)
constexpr int TH_LINE = 3;   // line search
constexpr int TH_TAIL = 4;   // remaining SSI budget

template <int NC>
struct ThreeLane
{
    static constexpr int M = 2 * NC;
    int mode, it, ssiSteps, newtonIt, col, side, ls, total;
    double P, T;
    double z[NC];
    double kg[NC], kw[NC];
    double logK[M];
    double bg, bw, damping;
    double J[M][M];
    double delta[M];
    ThreePhaseLogKState<NC> base;
    Result<NC> r;
};

template <int NC>
NZ_HD void threeEnterTail(ThreeLane<NC> &L)
{
    L.it = L.ssiSteps;
    L.mode = TH_TAIL;
}

template <int NC>
NZ_HD void threeEnterNewton(ThreeLane<NC> &L)
{
    for (int i = 0; i < NC; ++i)
    {
        L.logK[i] = log(L.kg[i]);
        L.logK[NC + i] = log(L.kw[i]);
    }
    L.newtonIt = 0;
    L.mode = TH_BASE;
}

template <int NC>
NZ_HD void threeInit(Solver<NC> &s, ThreeLane<NC> &L, const double *kgIn, const double *kwIn)
{
    L.r.init();
    L.r.presence = ALL_BITS;
    for (int i = 0; i < NC; ++i)
    {
        L.kg[i] = sclamp(kgIn[i], 1.0e-100, 1.0e100);
        L.kw[i] = sclamp(kwIn[i], 1.0e-100, 1.0e100);
    }
    L.bg = 0.15;
    L.bw = 0.15;
    L.ssiSteps = imin(s.O().maxIterations, imax(s.O().threeSsi, 0));
    L.total = 0;
    L.it = 0;
    L.mode = TH_SSI;
    if (L.ssiSteps == 0)
        threeEnterNewton(L);
}

// One step.  Returns 1 when the solve has ended: L.r is flashThree's result
// (and s.err may be set).
template <int NC>
NZ_HD int threeStep(Solver<NC> &s, ThreeLane<NC> &L)
{
    constexpr int M = 2 * NC;
    switch (L.mode)
    {
    case TH_SSI:
        if (!s.threeSsiStep(L.P, L.T, L.z, L.kg, L.kw, L.bg, L.bw, L.total, L.r))
            return 1;
        if (L.r.converged || s.err)
            return 1;
        if (++L.it >= L.ssiSteps)
            threeEnterNewton(L);
        return 0;
    case TH_BASE:
        if (L.newtonIt >= s.O().threeNewton)
        {
            threeEnterTail(L);
            return 0;
        }
        s.evalThree(L.P, L.T, L.z, L.logK, L.bg, L.bw, L.base);
        if (!L.base.valid || s.err)
        {
            threeEnterTail(L);
            return 0;
        }
        L.r = L.base.result;
        L.r.iterations = ++L.total;
        L.bg = L.r.beta[1];
        L.bw = L.r.beta[2];
        if (L.base.norm < s.O().fugacityTol)
        {
            L.r.converged = true;
            L.r.presence = s.presenceFromFractions(L.r.beta);
            s.updateSaturations(L.P, L.T, L.r);
            return 1;
        }
        L.col = 0;
        L.side = 1;
        L.mode = TH_FD;
        return 0;
    case TH_FD:
    {
        const double step = s.O().fdStep * smax(1.0, fabs(L.logK[L.col]));
        double pert[M];
        for (int i = 0; i < M; ++i)
            pert[i] = L.logK[i];
        if (L.side > 0)
            pert[L.col] += step;
        else
            pert[L.col] -= step;
        ThreePhaseLogKState<NC> probe;
        s.evalThree(L.P, L.T, L.z, pert, L.bg, L.bw, probe);
        if (L.side > 0)
        {
            if (!probe.valid)
            {
                L.side = -1;
                return 0;
            }
            for (int row = 0; row < M; ++row)
                L.J[row][L.col] = (probe.residual[row] - L.base.residual[row]) / step;
        }
        else
        {
            if (!probe.valid)
            {
                threeEnterTail(L);
                return 0;
            }
            for (int row = 0; row < M; ++row)
                L.J[row][L.col] = (L.base.residual[row] - probe.residual[row]) / step;
        }
        L.side = 1;
        if (++L.col < M)
            return 0;
        double rhs[M];
        for (int i = 0; i < M; ++i)
            rhs[i] = -L.base.residual[i];
        if (!solveDense<M>(L.J, rhs, L.delta))
        {
            threeEnterTail(L);
            return 0;
        }
        L.damping = 1.0;
        L.ls = 0;
        L.mode = TH_LINE;
        return 0;
    }
    case TH_LINE:
    {
        double trial[M];
        for (int i = 0; i < M; ++i)
            trial[i] = L.logK[i] + L.damping * L.delta[i];
        ThreePhaseLogKState<NC> probe;
        s.evalThree(L.P, L.T, L.z, trial, L.bg, L.bw, probe);
        if (probe.valid && probe.norm < L.base.norm)
        {
            for (int i = 0; i < M; ++i)
                L.logK[i] = trial[i];
            ++L.newtonIt;
            L.mode = TH_BASE;
            return 0;
        }
        L.damping *= 0.5;
        if (++L.ls >= 16)
            threeEnterTail(L);
        return 0;
    }
    default:   // TH_TAIL
        if (L.it >= s.O().maxIterations || s.err)
            return 1;
        for (int i = 0; i < NC; ++i)
        {
            L.kg[i] = exp(sclamp(L.logK[i], -230.0, 230.0));
            L.kw[i] = exp(sclamp(L.logK[NC + i], -230.0, 230.0));
        }
        if (!s.threeSsiStep(L.P, L.T, L.z, L.kg, L.kw, L.bg, L.bw, L.total, L.r))
            return 1;
        if (L.r.converged)
            return 1;
        for (int i = 0; i < NC; ++i)
        {
            L.logK[i] = log(L.kg[i]);
            L.logK[NC + i] = log(L.kw[i]);
        }
        ++L.it;
        return 0;
    }
}

} // namespace nz
