// staged_kernels.cuh -- kernels and launcher of the staged batched flash.
#pragma once

#include "common.cuh"
#include "staged.cuh"

#include <cstdio>
#include <cstdlib>

namespace nz
{

template <int NC>
NZ_HDI void writeFlashOut(const nz_flash_out &out, int64_t n, int64_t i, const Result<NC> &r, uint8_t status)
{
    if (out.status) out.status[i] = status;
    if (out.presence) out.presence[i] = (r.converged && status == NZ_FLASH_CONVERGED) ? r.presence : 0;
    if (out.iterations) out.iterations[i] = r.iterations;
    for (int p = 0; p < 3; ++p)
    {
        if (out.beta) out.beta[p * n + i] = r.beta[p];
        if (out.saturation) out.saturation[p * n + i] = r.sat[p];
        if (out.compressibility) out.compressibility[p * n + i] = r.Z[p];
        if (out.molar_density) out.molar_density[p * n + i] = r.rho[p];
        if (out.composition)
            for (int c = 0; c < NC; ++c)
                out.composition[(p * NC + c) * n + i] = r.x[p][c];
    }
    for (int c = 0; c < NC; ++c)
    {
        if (out.k_gas_oil) out.k_gas_oil[c * n + i] = r.Kg[c];
        if (out.k_water_oil) out.k_water_oil[c * n + i] = r.Kw[c];
    }
}

__device__ __forceinline__ void warpAddEvals(unsigned long long *counter, unsigned long long v)
{
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v)
        atomicAdd(counter, v);
}

// NZ_STAGED_SYNC=1 synchronises after every staged launch and reports the
// queue counters and self-check words (debugging aid; off by default).
inline bool stagedDebugSync()
{
    static const bool on = [] {
        const char *v = std::getenv("NZ_STAGED_SYNC");
        return v != nullptr && v[0] == '1';
    }();
    return on;
}

struct StagedArgs
{
    int64_t n;
    const double *P;
    const double *T;
    const double *z;
    const double *sal;
    void *states;             // DriverState<NC>[n]
    void *trials;             // TrialOut<NC>[n * 3 * nseeds]
    unsigned long long *tasks[2];
    int *pending[2];
    int *full;
    int *split[2];            // resumed points: [0] finish directly, [1] continue with a new phase set
    int *counters;            // per round r: [4r]=tasks [4r+1]=pending [4r+2]=trial cursor [4r+3]=split0;
                              // rounds kMaxRounds.. are the recovery rounds; then full, bound flag,
                              // guard flag, split1 of the current round, continuation queue, rest queue
    unsigned long long *threes;   // three-phase solves: (point << 1) | kind (0 active-set path, 1 recovery 1)
    unsigned long long *threesLong;   // solves past the lane budget, for the warp kernel (same encoding)
    int *cont;                // points queued for the pressure continuation
    void *anchors;            // AnchorOut<NC>[contCap * 8]
    int64_t contCap;
    unsigned long long *evalCounter;
    int mixed;   // TPD trials: mixed-precision leading SSI steps
    // Multi-model batches: the fluid of each model and the model of each point
    // (null: every point uses the kernels' own fluid argument).
    const FluidDev *fluids;
    const uint16_t *model;
    // SW allocation search ahead of the recovery kernel (SW batches only):
    // AllocMemo<NC>[allocCap] and the point of each memo slot
    void *allocMemos;
    int *allocPoints;
    int64_t allocCap;
    // the role-permutation searches of the same points (PermMemo<NC>[allocCap],
    // indexed by the allocation slot) and the slots queued for them
    void *permMemos;
    int *permSlots;
};

// The fluid point i is flashed with, and its salinity.
__device__ __forceinline__ const FluidDev *pointFluid(const FluidDev &F, const StagedArgs &a, int64_t i)
{
    return a.fluids ? a.fluids + a.model[i] : &F;
}
__device__ __forceinline__ double pointSalinity(const FluidDev &F, const StagedArgs &a, int64_t i)
{
    return a.sal ? a.sal[i] : pointFluid(F, a, i)->salinity;
}

// Per-round counters for the active-set rounds and the recovery rounds, then
// the shared ones.
constexpr int kRecoveryRounds = 3;   // stableReducedSetFallback_: one stability test per candidate pair
constexpr int kRoundSlots = kMaxRounds + kRecoveryRounds;
constexpr int kCounterFull = 4 * kRoundSlots;
constexpr int kCounterBound = kCounterFull + 1;
constexpr int kCounterGuard = kCounterFull + 2;
constexpr int kCounterSplit1 = kCounterFull + 3;
constexpr int kCounterCont = kCounterFull + 4;
constexpr int kCounterRest = kCounterFull + 5;
constexpr int kCounterThree = kCounterFull + 6;        // queued three-phase solves
constexpr int kCounterThreeCursor = kCounterFull + 7;  // refill cursor of the three-phase kernel
constexpr int kCounterThreeLong = kCounterFull + 8;    // solves handed to the warp kernel
constexpr int kCounterAlloc = kCounterFull + 9;        // points queued for the lane allocation search
constexpr int kCounterAllocCursor = kCounterFull + 10; // its (point, seed) task cursor
constexpr int kCounterPerm = kCounterFull + 11;        // points queued for the warp permutation search
// Steps a lane of the three-phase kernel gives one solve before handing it to
// the warp kernel.  Most solves end within ~40 steps; the few long ones are
// long because their robust Rachford-Rice solves fail start after start,
// which the warp kernel runs on parallel lanes.
constexpr int kThreeLaneSteps = 48;
constexpr int kCounterWords = kCounterFull + 12;
constexpr int kAnchors = 8;

// Result of one pressure-continuation anchor of one point.
template <int NC>
struct AnchorOut
{
    int outcome;   // CONT_NONE / CONT_SUCCESS / CONT_ERROR
    int err;
    Result<NC> r;
};

// Points whose pressure continuation runs on the anchor kernels (one warp per
// anchor); beyond this the recovery kernel runs it in place, anchor by anchor.
inline int64_t contCapacity(int64_t n)
{
    if (n <= 64)
        return n;
    return n / 32 < 64 ? 64 : n / 32;
}

// Memo slots of the lane allocation search (SW batches): an eighth of the
// points (the search is reached by ~7 % of a typical SW batch); points past it
// run the search inside the recovery kernel.
inline int64_t allocCapacity(int64_t n, const FluidDev &F)
{
    if (F.eosModel != EOS_SW)
        return 0;
    const int64_t cap = n / 8 + 256;
    return cap < n ? cap : n;
}

// A queue bound or a spin guard has tripped in this batch: the kernels that
// follow leave the unfinished points alone (their status stays
// NZ_FLASH_UNFINISHED) instead of building on incomplete queues.  The test is
// warp-uniform (read at kernel entry with every lane of the warp active), so a
// warp leaves as a whole and no lane waits at a warp-wide operation.
__device__ __forceinline__ bool stagedTripped(const StagedArgs &a)
{
    const bool tripped = a.counters[kCounterBound] != 0 || a.counters[kCounterGuard] != 0;
    return __any_sync(0xffffffffu, tripped);
}

// After the last kernel of a batch: copy its queue-bound and spin-guard codes
// to `sink` ([0] bound, [1] guard; the context's check words), if given.
static __global__ void stagedCheckKernel(const int *counters, int *sink)
{
    if (threadIdx.x == 0 && blockIdx.x == 0 && sink)
    {
        sink[0] = counters[kCounterBound];
        sink[1] = counters[kCounterGuard];
    }
}

// Dispatch a point after its driver returned.
template <int NC>
__device__ void routePoint(const StagedArgs &a, const nz_flash_out &out, int round, int64_t i, uint8_t stage,
                           Driver<NC> &d)
{
    DriverState<NC> &st = *d.st;
    st.err = d.s.err;
    if (stage == STAGE_DONE)
        stage = d.finish();
    if (stage == STAGE_NEED_STABILITY && round + 1 >= kMaxRounds)
        stage = STAGE_NEED_FULL;
    st.stage = stage;
    if (stage == STAGE_DONE)
    {
        writeFlashOut<NC>(out, a.n, i, st.current, NZ_FLASH_CONVERGED);
    }
    else if (stage == STAGE_NEED_THREE)
    {
        const int k = atomicAdd(&a.counters[kCounterThree], 1);
        if (k < a.n)
            a.threes[k] = static_cast<unsigned long long>(i) << 1;
        else
            atomicExch(&a.counters[kCounterBound], 13);
    }
    else if (stage == STAGE_NEED_FULL)
    {
        const int k = atomicAdd(&a.counters[kCounterFull], 1);
        if (k < a.n)
            a.full[k] = int(i);
        else
            atomicExch(&a.counters[kCounterBound], 1);
    }
    else
    {
        const int q = round & 1;
        const int k = atomicAdd(&a.counters[4 * round + 1], 1);
        if (k < a.n && round < kMaxRounds)
            a.pending[q][k] = int(i);
        else
            atomicExch(&a.counters[kCounterBound], 2);
        for (int cand = 0; cand < 3; ++cand)
            if (!(st.tested & bitOf(cand)))
            {
                const int t = atomicAdd(&a.counters[4 * round], 1);
                if (t < 3 * a.n)
                    a.tasks[q][t] = (static_cast<unsigned long long>(i) << 2) | unsigned(cand);
                else
                    atomicExch(&a.counters[kCounterBound], 3);
            }
    }
}

template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedStartKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                  const __grid_constant__ nz_flash_out out)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    unsigned long long evals = 0;
    if (i < a.n)
    {
        // final statuses overwrite this; a point a tripped self-check leaves keeps it
        if (out.status)
            out.status[i] = NZ_FLASH_UNFINISHED;
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        Driver<NC> d;
        d.st = &states[i];
        const double sal = pointSalinity(F, a, i);
        d.s.setup(pointFluid(F, a, i), sal);
        d.st->sal = sal;
        double zi[NC];
        for (int c = 0; c < NC; ++c)
            zi[c] = a.z[c * a.n + i];
        uint8_t stage = d.start(a.P[i], a.T[i], zi);
        if (stage == STAGE_DONE)
            stage = d.activeSetLoop(false, nullptr);
        routePoint<NC>(a, out, 0, i, stage, d);
        evals = d.s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

// Combine each pending point's trials into its stability result and sort the
// points by what comes next, so the warps of the resume launches are uniform:
// [0] the test ends the active-set loop (stable / invalid), [1] phases are
// added and a new equilibrium follows.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedClassifyKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a, int round)
{
    if (stagedTripped(a))
        return;
    const int q = round & 1;
    const int count = a.counters[4 * round + 1];
    const int nseeds = seedCount<NC>(F);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count && k < a.n; k += gridDim.x * blockDim.x)
    {
        const int64_t i = a.pending[q][k];
        if (i < 0 || i >= a.n)
        {
            atomicExch(&a.counters[kCounterBound], 4);
            continue;
        }
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        const TrialOut<NC> *trials = static_cast<const TrialOut<NC> *>(a.trials) + i * 3 * nseeds;
        Driver<NC> d;
        d.st = &states[i];
        d.s.setup(pointFluid(F, a, i), d.st->sal);
        d.combineStability(trials, nseeds, d.st->sr);
        d.st->err = d.s.err;   // a trial error ends the active-set path on resume
        bool adds = false;
        if (d.st->sr.valid && !d.st->sr.stable)
            for (int p = 0; p < 3; ++p)
                adds = adds || (!(d.st->tested & bitOf(p)) && d.st->sr.unstable[p]);
        const int which = adds ? 1 : 0;
        const int slot = atomicAdd(which ? &a.counters[kCounterSplit1] : &a.counters[4 * round + 3], 1);
        if (slot < a.n)
            a.split[which][slot] = int(i);
        else
            atomicExch(&a.counters[kCounterBound], 7);
    }
}

template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedResumeKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                   const __grid_constant__ nz_flash_out out, int round, int which)
{
    if (stagedTripped(a))
        return;
    const int count = which ? a.counters[kCounterSplit1] : a.counters[4 * round + 3];
    unsigned long long evals = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count && k < a.n; k += gridDim.x * blockDim.x)
    {
        const int64_t i = a.split[which][k];
        if (i < 0 || i >= a.n)
        {
            atomicExch(&a.counters[kCounterBound], 4);
            continue;
        }
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        Driver<NC> d;
        d.st = &states[i];
        d.s.setup(pointFluid(F, a, i), d.st->sal);
        d.s.err = d.st->err;
        const StabilityResult<NC> sr = d.st->sr;
        const uint8_t stage = d.activeSetLoop(true, &sr);
        routePoint<NC>(a, out, round + 1, i, stage, d);
        evals += d.s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

// The split-1 and three-phase counters are shared by the rounds; reset them between them.
static __global__ void stagedResetSplitKernel(int *counters)
{
    counters[kCounterSplit1] = 0;
    counters[kCounterThree] = 0;
    counters[kCounterThreeCursor] = 0;
    counters[kCounterThreeLong] = 0;
}

// Every queued three-phase solve is a lane running flashThree_ one step at a
// time (ThreeLane); idle lanes are refilled with one atomic per warp.  The
// result goes to the point's current (active-set path) or lastPhysical
// (recovery 1) record.
template <int NC>
__global__ void __launch_bounds__(kTrialBlock)
stagedThreeKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a)
{
    if (stagedTripped(a))
        return;
    const int queued = a.counters[kCounterThree];
    const long long total = queued < a.n ? queued : a.n;
    int *cursor = &a.counters[kCounterThreeCursor];
    DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
    const int nseeds = seedCount<NC>(F);
    const unsigned lane = threadIdx.x & 31;
    Solver<NC> s;
    s.setup(&F, 0.0);
    ThreeLane<NC> L;
    long long point = -1;   // -1 idle, -2 drained
    int kind = 0;
    int steps = 0;
    unsigned long long evals = 0;
    // a solve takes at most ssi + newton * (1 + 4 nc + 16) + tail steps (a few
    // hundred); the cap only guards against a wait that would never end
    long long guard = 0;
    const long long guardMax = F.spinLimit;
    while (true)
    {
        if (++guard > guardMax)
        {
            atomicExch(&a.counters[kCounterGuard], 2);
            break;
        }
        const bool need = point == -1;
        const unsigned mask = __ballot_sync(0xffffffffu, need);
        if (mask)
        {
            int base = 0;
            if (lane == unsigned(__ffs(mask) - 1))
                base = atomicAdd(cursor, __popc(mask));
            base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
            if (need)
            {
                const long long idx = base + __popc(mask & ((1u << lane) - 1u));
                if (idx < total)
                {
                    const unsigned long long task = a.threes[idx];
                    const int64_t i = int64_t(task >> 1);
                    if (i < 0 || i >= a.n)
                    {
                        atomicExch(&a.counters[kCounterBound], 14);
                        point = -2;
                    }
                    else
                    {
                        const DriverState<NC> &st = states[i];
                        evals += s.evals;
                        s.setup(pointFluid(F, a, i), st.sal);
                        kind = int(task & 1u);
                        if (kind == 1)
                            s.memo = reinterpret_cast<const Rr3Memo<NC> *>(static_cast<const TrialOut<NC> *>(a.trials) +
                                                                            i * 3 * nseeds);
                        L.P = st.P;
                        L.T = st.T;
                        for (int c = 0; c < NC; ++c)
                            L.z[c] = st.z[c];
                        threeInit<NC>(s, L, st.threeKg, st.threeKw);
                        point = i;
                        steps = 0;
                    }
                }
                else
                {
                    point = -2;
                }
            }
        }
        const bool running = point >= 0;
        if (!__any_sync(0xffffffffu, running))
            break;
        if (!running)
            continue;
        if (steps >= kThreeLaneSteps)
        {
            // over budget: the warp kernel solves it again from the start
            const int k = atomicAdd(&a.counters[kCounterThreeLong], 1);
            if (k >= 0 && k < a.n)
            {
                a.threesLong[k] = (static_cast<unsigned long long>(point) << 1) | unsigned(kind);
                s.err = ERR_NONE;
                point = -1;
                continue;
            }
        }
        ++steps;
        if (threeStep<NC>(s, L))
        {
            DriverState<NC> &st = states[point];
            if (kind == 1)
                st.lastPhysical = L.r;
            else
                st.current = L.r;
            st.err = s.err;
            point = -1;
        }
    }
    evals += s.evals;
    warpAddEvals(a.evalCounter, evals);
}

// The solves the lane kernel handed over: a warp per solve runs flashThree_
// from its start with the robust Rachford-Rice starts split over the lanes
// (Solver::rr3Robust's warp path), which is the same solve.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedThreeLongKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a)
{
    if (stagedTripped(a))
        return;
    const int queued = a.counters[kCounterThreeLong];
    const int64_t count = queued < a.n ? queued : a.n;
    const int lane = threadIdx.x & 31;
    const int64_t warpId = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int nseeds = seedCount<NC>(F);
    DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
    unsigned long long evals = 0;
    for (int64_t k = warpId; k < count; k += nwarps)
    {
        const unsigned long long task = a.threesLong[k];
        const int64_t i = int64_t(task >> 1);
        if (i < 0 || i >= a.n)
        {
            if (lane == 0)
                atomicExch(&a.counters[kCounterBound], 15);
            continue;
        }
        DriverState<NC> &st = states[i];
        const int kind = int(task & 1u);
        Solver<NC> s;
        s.setup(pointFluid(F, a, i), st.sal);
        s.lane = lane;
        s.width = 32;
        if (kind == 1)
            s.memo = reinterpret_cast<const Rr3Memo<NC> *>(static_cast<const TrialOut<NC> *>(a.trials) +
                                                            i * 3 * nseeds);
        double kg[NC], kw[NC];
        for (int c = 0; c < NC; ++c)
        {
            kg[c] = st.threeKg[c];
            kw[c] = st.threeKw[c];
        }
        Result<NC> r;
        s.flashThree(st.P, st.T, st.z, kg, kw, r);
        __syncwarp();
        if (lane == 0)
        {
            if (kind == 1)
                st.lastPhysical = r;
            else
                st.current = r;
            st.err = s.err;
            evals += s.evals;
        }
    }
    warpAddEvals(a.evalCounter, evals);
}

// Active-set points whose three-phase solve is done: resume their loop.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedThreeResumeKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                        const __grid_constant__ nz_flash_out out, int round)
{
    if (stagedTripped(a))
        return;
    const int queued = a.counters[kCounterThree];
    const int count = queued < a.n ? queued : int(a.n);
    unsigned long long evals = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
    {
        const unsigned long long task = a.threes[k];
        const int64_t i = int64_t(task >> 1);
        if (i < 0 || i >= a.n || (task & 1u))
            continue;
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        Driver<NC> d;
        d.st = &states[i];
        d.s.setup(pointFluid(F, a, i), d.st->sal);
        d.s.err = d.st->err;
        const uint8_t stage = d.activeSetLoop(false, nullptr, true);
        routePoint<NC>(a, out, round + 1, i, stage, d);
        evals += d.s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

// Every (task, seed) TPD trial is a lane; idle lanes are refilled from the
// round's task list with one atomic per warp.
// A TrialOut slot holding a trial's state after the mixed form's FP32 phase
// (x = ln W, sum = steps done, trivial = mode) rather than a result.
constexpr int kTrialMixedContinue = 0x4d495844;

// The mixed form's FP32 phase of every queued trial of this round, thread per
// trial (trialMixedPhase: at most the leading SSI budget of
// FP32 steps), ahead of stagedTrialKernel, which then runs every later step
// in FP64 -- so the FP64 kernel carries no FP32 code.
template <int NC>
__global__ void __launch_bounds__(kTrialBlock)
stagedTrialMixedKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a, int round)
{
    if (stagedTripped(a))
        return;
    const int q = round & 1;
    const int nseeds = seedCount<NC>(F);
    const int ntasks = a.counters[4 * round];
    const long long total = static_cast<long long>(ntasks < 3 * a.n ? ntasks : 3 * a.n) * nseeds;
    const DriverState<NC> *states = static_cast<const DriverState<NC> *>(a.states);
    TrialOut<NC> *trials = static_cast<TrialOut<NC> *>(a.trials);
    unsigned long long evals = 0;
    Solver<NC> s;
    TrialLane<NC> L;
    for (long long idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += int64_t(gridDim.x) * blockDim.x)
    {
        const unsigned long long task = a.tasks[q][idx / nseeds];
        const int seedIndex = int(idx % nseeds);
        const int64_t point = int64_t(task >> 2);
        const int cand = int(task & 3u);
        if (point < 0 || point >= a.n || cand > 2)
            continue;   // the trial kernel reports it
        const DriverState<NC> &st = states[point];
        s.setup(pointFluid(F, a, point), st.sal);
        s.mixed = true;
        L.P = st.P;
        L.T = st.T;
        L.candidate = cand;
        for (int c = 0; c < NC; ++c)
        {
            L.logRef[c] = st.logRef[c];
            L.ref[c] = st.refX[c];
        }
        double seed[NC];
        s.stabilitySeed(seedIndex, st.P, st.T, st.z, st.refX, seed);
        trialInit<NC>(s, L, seed);
        const int rc = trialMixedPhase<NC>(s, L);
        TrialOut<NC> &o = trials[(point * 3 + cand) * nseeds + seedIndex];
        if (rc != 0 || s.err)
        {
            o.valid = s.err ? -s.err : 0;
            o.trivial = 0;
            o.sum = 0.0;
            for (int c = 0; c < NC; ++c)
                o.x[c] = 0.0;
        }
        else
        {
            o.valid = kTrialMixedContinue;
            o.trivial = L.mode;
            o.sum = double(L.it);
            for (int c = 0; c < NC; ++c)
                o.x[c] = L.logW[c];
        }
        evals += s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

template <int NC>
__global__ void __launch_bounds__(kTrialBlock)
stagedTrialKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a, int round)
{
    if (stagedTripped(a))
        return;
    const int q = round & 1;
    const int nseeds = seedCount<NC>(F);
    const int ntasks = a.counters[4 * round];
    const long long total = static_cast<long long>(ntasks < 3 * a.n ? ntasks : 3 * a.n) * nseeds;
    int *cursor = &a.counters[4 * round + 2];
    const DriverState<NC> *states = static_cast<const DriverState<NC> *>(a.states);
    TrialOut<NC> *trials = static_cast<TrialOut<NC> *>(a.trials);
    const unsigned lane = threadIdx.x & 31;

    Solver<NC> s;
    s.setup(&F, 0.0);
    TrialLane<NC> L;
    long long slot = -1;       // output slot of the running trial, -1 idle, -2 drained
    unsigned long long evals = 0;
    // A trial takes at most ~8 + 12*(NC+17) + 72 steps; a warp runs its
    // lanes' trials back to back, so this cap is far above any real need and
    // only guards against a wait that would never end.
    long long guard = 0;
    const long long guardMax = F.spinLimit;
    while (true)
    {
        if (++guard > guardMax)
        {
            atomicExch(&a.counters[kCounterGuard], 1);
            break;
        }
        const bool need = slot == -1;
        const unsigned mask = __ballot_sync(0xffffffffu, need);
        if (mask)
        {
            int base = 0;
            if (lane == unsigned(__ffs(mask) - 1))
                base = atomicAdd(cursor, __popc(mask));
            base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
            if (need)
            {
                const long long idx = base + __popc(mask & ((1u << lane) - 1u));
                if (idx < total)
                {
                    const unsigned long long task = a.tasks[q][idx / nseeds];
                    const int seedIndex = int(idx % nseeds);
                    const int64_t point = int64_t(task >> 2);
                    const int cand = int(task & 3u);
                    const bool bad = point < 0 || point >= a.n || cand > 2;
                    if (bad)
                        atomicExch(&a.counters[kCounterBound], 5);
                    const DriverState<NC> &st = states[bad ? 0 : point];
                    evals += s.evals;
                    s.setup(pointFluid(F, a, bad ? 0 : point), st.sal);
                    L.P = st.P;
                    L.T = st.T;
                    L.candidate = cand;
                    for (int c = 0; c < NC; ++c)
                    {
                        L.logRef[c] = st.logRef[c];
                        L.ref[c] = st.refX[c];
                    }
                    double seed[NC];
                    s.stabilitySeed(seedIndex, st.P, st.T, st.z, st.refX, seed);
                    trialInit<NC>(s, L, seed);
                    slot = bad ? -2 : (point * 3 + cand) * nseeds + seedIndex;
                    if (a.mixed && !bad)
                    {
                        // the mixed form's FP32 phase ran ahead (stagedTrialMixedKernel):
                        // continue from its state, or leave a trial it ended
                        const TrialOut<NC> &pre = trials[slot];
                        if (pre.valid == kTrialMixedContinue)
                        {
                            for (int c = 0; c < NC; ++c)
                                L.logW[c] = pre.x[c];
                            L.it = int(pre.sum);
                            L.mode = pre.trivial;
                            L.fp64Ssi = true;
                        }
                        else
                            slot = -1;
                    }
                }
                else
                {
                    slot = -2;
                }
            }
        }
        const bool running = slot >= 0;
        if (!__any_sync(0xffffffffu, running))
            break;
        if (running)
        {
            TrialOut<NC> res;
            const int rc = trialStep<NC>(s, L, res);
            if (rc != 0 || s.err)
            {
                if (rc != 1 || s.err)
                {
                    // an EOS error is kept (as -code): it aborts the test
                    res.valid = s.err ? -s.err : 0;
                    res.trivial = 0;
                    res.sum = 0.0;
                    for (int c = 0; c < NC; ++c)
                        res.x[c] = 0.0;
                }
                trials[slot] = res;
                slot = -1;
                s.err = ERR_NONE;
            }
        }
    }
    evals += s.evals;
    warpAddEvals(a.evalCounter, evals);
}

// solveRr3_ (nonlinear.inc:8-96) with the line search spread over a warp: the
// sequential loop tries lambda = 2^-l for l = 0, 1, ... 39 and takes the first
// that lowers the norm; here lane l (and l + 32) evaluates 2^-l at once and the
// lowest accepted l wins, which is the same step.
template <int NC>
__device__ bool rr3Warp(const Solver<NC> &s, const double *z, const double *kg, const double *kw, double initBg,
                        double initBw, double &outBg, double &outBw)
{
    const int lane = threadIdx.x & 31;
    double bg = sclamp(initBg, 1.0e-4, 0.8);
    double bw = sclamp(initBw, 1.0e-4, 0.8);
    if (bg + bw >= 0.95)
    {
        const double scale = 0.8 / (bg + bw);
        bg *= scale;
        bw *= scale;
    }
    for (int it = 0; it < s.O().maxRr; ++it)
    {
        double fg, fw, jgg, jww, jgw;
        const double norm = s.rr3Norm(z, kg, kw, bg, bw, fg, fw, jgg, jww, jgw);
        if (!isfinite(norm))
            return false;
        if (norm < s.O().rrTol)
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
        bool accepted = false;
        for (int base = 0; base < 40 && !accepted; base += 32)
        {
            const int l = base + lane;
            bool ok = false;
            double cg = 0.0, cw = 0.0;
            if (l < 40)
            {
                const double lambda = ldexp(1.0, -l);
                cg = bg + lambda * dbg;
                cw = bw + lambda * dbw;
                double a, b, c, d, e;
                const double cn = s.rr3Norm(z, kg, kw, cg, cw, a, b, c, d, e);
                ok = isfinite(cn) && cn < norm;
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (m)
            {
                const int src = __ffs(m) - 1;
                bg = __shfl_sync(0xffffffffu, cg, src);
                bw = __shfl_sync(0xffffffffu, cw, src);
                accepted = true;
            }
        }
        if (!accepted)
            return false;
    }
    return false;
}

// The first robust RR3 of recovery 1 (flashThree from Wilson K_g and the
// initial K_w, fractions 0.15 / 0.15), one warp per point, starts in
// solveRr3Robust_'s order.  The answer is kept as the point's Rr3Memo, in its
// trial slots (unused until recovery 2 queues trials).
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedRr3MemoKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a)
{
    if (stagedTripped(a))
        return;
    const int count = a.counters[kCounterFull];
    const int nseeds = seedCount<NC>(F);
    const int lane = threadIdx.x & 31;
    const int64_t warpId = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const double guesses[17][2] = {
        {0.15, 0.15}, {0.333, 0.333}, {0.50, 1.0e-4}, {1.0e-4, 0.50}, {0.80, 1.0e-4},
        {1.0e-4, 0.80}, {0.20, 0.20}, {0.60, 0.20}, {0.20, 0.60}, {0.05, 0.05},
        {0.90, 0.01}, {0.95, 1.0e-4}, {0.98, 1.0e-4}, {1.0e-4, 0.95}, {1.0e-4, 0.98},
        {0.01, 0.90}, {0.45, 0.45}};
    for (int64_t k = warpId; k < count && k < a.n; k += nwarps)
    {
        const int64_t i = a.full[k];
        if (i < 0 || i >= a.n)
            continue;
        const DriverState<NC> &st = static_cast<const DriverState<NC> *>(a.states)[i];
        if (!st.mainFailed)
            continue;
        Solver<NC> s;
        s.setup(pointFluid(F, a, i), st.sal);
        Rr3Memo<NC> m;
        double kg[NC], kw[NC];
        s.wilsonK(st.P, st.T, kg);
        s.initialWaterK(kw);
        for (int c = 0; c < NC; ++c)
        {
            m.z[c] = st.z[c];
            m.kg[c] = sclamp(kg[c], 1.0e-100, 1.0e100);
            m.kw[c] = sclamp(kw[c], 1.0e-100, 1.0e100);
        }
        m.pg = m.pw = 0.15;
        m.ok = 0;
        m.bg = m.bw = 0.0;
        for (int g = 0; g < 17 && !m.ok; ++g)
            m.ok = rr3Warp<NC>(s, m.z, m.kg, m.kw, g == 0 ? m.pg : guesses[g][0], g == 0 ? m.pw : guesses[g][1],
                               m.bg, m.bw) ? 1 : 0;
        m.valid = 1;
        if (lane == 0)
            *reinterpret_cast<Rr3Memo<NC> *>(static_cast<TrialOut<NC> *>(a.trials) + i * 3 * nseeds) = m;
    }
}

// Where a point goes after a recovery step (recovery rounds are numbered from
// kMaxRounds): more trials, an answer, an error, or the warp recovery kernel.
template <int NC>
__device__ void routeRecovery(const StagedArgs &a, const nz_flash_out &out, int rr, int64_t i, uint8_t stage,
                              Driver<NC> &d)
{
    DriverState<NC> &st = *d.st;
    if (stage == STAGE_NEED_STABILITY && rr < kRecoveryRounds)
    {
        const int round = kMaxRounds + rr;
        const int q = round & 1;
        const int k = atomicAdd(&a.counters[4 * round + 1], 1);
        if (k < a.n)
            a.pending[q][k] = int(i);
        else
            atomicExch(&a.counters[kCounterBound], 9);
        for (int cand = 0; cand < 3; ++cand)
            if (!(st.tested & bitOf(cand)))
            {
                const int t = atomicAdd(&a.counters[4 * round], 1);
                if (t < 3 * a.n)
                    a.tasks[q][t] = (static_cast<unsigned long long>(i) << 2) | unsigned(cand);
                else
                    atomicExch(&a.counters[kCounterBound], 10);
            }
        return;
    }
    if (stage == STAGE_NEED_STABILITY)   // more pairs than rounds: cannot happen (3 pairs, 3 rounds)
        atomicExch(&a.counters[kCounterBound], 11);
    if (d.s.err)
    {
        Result<NC> failed;
        failed.init();
        writeFlashOut<NC>(out, a.n, i, failed, uint8_t(d.s.err));
        return;
    }
    if (d.reducedFinish())
    {
        if (d.s.err)
        {
            Result<NC> failed;
            failed.init();
            writeFlashOut<NC>(out, a.n, i, failed, uint8_t(d.s.err));
        }
        else
            writeFlashOut<NC>(out, a.n, i, st.current, NZ_FLASH_CONVERGED);
        return;
    }
    st.recoverFrom = 3;
    const int k = atomicAdd(&a.counters[kCounterRest], 1);
    if (k < a.n)
        a.split[0][k] = int(i);
    else
        atomicExch(&a.counters[kCounterBound], 12);
}

// Points whose active-set path failed: flash()'s recovery 1, then recovery 2
// up to its first stability test.  Points that failed for another reason
// (an error, too many rounds) go to the warp recovery kernel whole.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedRecoverStartKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                         const __grid_constant__ nz_flash_out out)
{
    if (stagedTripped(a))
        return;
    const int count = a.counters[kCounterFull];
    unsigned long long evals = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count && k < a.n; k += gridDim.x * blockDim.x)
    {
        const int64_t i = a.full[k];
        if (i < 0 || i >= a.n)
        {
            atomicExch(&a.counters[kCounterBound], 6);
            continue;
        }
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        Driver<NC> d;
        d.st = &states[i];
        if (!d.st->mainFailed)
        {
            d.st->recoverFrom = 0;
            const int r = atomicAdd(&a.counters[kCounterRest], 1);
            if (r < a.n)
                a.split[0][r] = int(i);
            else
                atomicExch(&a.counters[kCounterBound], 12);
            continue;
        }
        d.s.setup(pointFluid(F, a, i), d.st->sal);
        d.recoveryOneStart();
        const int t = atomicAdd(&a.counters[kCounterThree], 1);
        if (t < a.n)
            a.threes[t] = (static_cast<unsigned long long>(i) << 1) | 1ull;
        else
            atomicExch(&a.counters[kCounterBound], 13);
        evals += d.s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

// Recovery 1's three-phase solve is done: accept it, or start recovery 2 up to
// its first stability test.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedRecoverThreeKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                         const __grid_constant__ nz_flash_out out)
{
    if (stagedTripped(a))
        return;
    const int queued = a.counters[kCounterThree];
    const int count = queued < a.n ? queued : int(a.n);
    unsigned long long evals = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
    {
        const unsigned long long task = a.threes[k];
        const int64_t i = int64_t(task >> 1);
        if (i < 0 || i >= a.n || !(task & 1u))
            continue;
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        Driver<NC> d;
        d.st = &states[i];
        d.s.setup(pointFluid(F, a, i), d.st->sal);
        d.s.err = d.st->err;
        Result<NC> full = d.st->lastPhysical;
        if (d.s.err || d.recoveryOneAccept(full))
        {
            if (d.s.err)
            {
                Result<NC> failed;
                failed.init();
                writeFlashOut<NC>(out, a.n, i, failed, uint8_t(d.s.err));
            }
            else
                writeFlashOut<NC>(out, a.n, i, d.st->current, NZ_FLASH_CONVERGED);
            evals += d.s.evals;
            continue;
        }
        d.st->seed.init();
        d.st->r2BestG = nzInf();
        d.st->r2Cand = 0;
        const uint8_t stage = d.reducedAdvance();
        routeRecovery<NC>(a, out, 0, i, stage, d);
        evals += d.s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

// Recovery round rr: certify the tested pair from its trials, then go on to
// the next pair.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedRecoverResumeKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                          const __grid_constant__ nz_flash_out out, int rr)
{
    if (stagedTripped(a))
        return;
    const int round = kMaxRounds + rr;
    const int q = round & 1;
    const int count = a.counters[4 * round + 1];
    const int nseeds = seedCount<NC>(F);
    unsigned long long evals = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count && k < a.n; k += gridDim.x * blockDim.x)
    {
        const int64_t i = a.pending[q][k];
        if (i < 0 || i >= a.n)
        {
            atomicExch(&a.counters[kCounterBound], 4);
            continue;
        }
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        const TrialOut<NC> *trials = static_cast<const TrialOut<NC> *>(a.trials) + i * 3 * nseeds;
        Driver<NC> d;
        d.st = &states[i];
        d.s.setup(pointFluid(F, a, i), d.st->sal);
        d.reducedCombine(trials, nseeds);
        const uint8_t stage = d.s.err ? STAGE_DONE : d.reducedAdvance();
        routeRecovery<NC>(a, out, rr + 1, i, stage, d);
        evals += d.s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

// Rest points whose next recovery is the SW allocation search get a memo
// slot, filled by stagedAllocSeedKernel before the recovery kernel runs;
// points past the capacity run the search inside the recovery kernel.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedAllocQueueKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a)
{
    if (stagedTripped(a))
        return;
    const int count = a.counters[kCounterRest];
    DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
    AllocMemo<NC> *memos = static_cast<AllocMemo<NC> *>(a.allocMemos);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count && k < a.n; k += gridDim.x * blockDim.x)
    {
        const int64_t i = a.split[0][k];
        if (i < 0 || i >= a.n)
        {
            atomicExch(&a.counters[kCounterBound], 16);
            continue;
        }
        DriverState<NC> &st = states[i];
        st.allocSlot = -1;
        if (st.recoverFrom != 3 || pointFluid(F, a, i)->eosModel != EOS_SW)
            continue;
        const int slot = atomicAdd(&a.counters[kCounterAlloc], 1);
        if (slot >= a.allocCap)
            continue;
        AllocMemo<NC> &m = memos[slot];
        m.P = a.P[i];
        m.T = a.T[i];
        m.salinity = st.sal;
        for (int c = 0; c < NC; ++c)
            m.z[c] = st.z[c];
        m.valid = 1;
        a.allocPoints[slot] = int(i);
        st.allocSlot = slot;
    }
}

// The queued allocation searches, one lane per (seed, point) task, tasks in
// seed-major order: every lane takes its next task with its own atomic -- a
// task is a whole preconditioning and refinement solve, so the lanes do not
// wait for one another -- and writes the seed's outcome into the point's memo.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedAllocSeedKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a)
{
    if (stagedTripped(a))
        return;
    const int queued = a.counters[kCounterAlloc];
    const int64_t points = queued < a.allocCap ? queued : a.allocCap;
    const int64_t total = points * kAllocSeedCount;
    const DriverState<NC> *states = static_cast<const DriverState<NC> *>(a.states);
    AllocMemo<NC> *memos = static_cast<AllocMemo<NC> *>(a.allocMemos);
    unsigned long long evals = 0;
    Solver<NC> s;
    while (true)
    {
        const int64_t t = atomicAdd(&a.counters[kCounterAllocCursor], 1);
        if (t >= total)
            break;
        // seed-major: consecutive lanes take the same seed of different
        // points, so a warp's lanes start in the same seed builder
        const int k = int(t / points);
        const int64_t slot = t % points;
        const int64_t i = a.allocPoints[slot];
        if (i < 0 || i >= a.n)
        {
            atomicExch(&a.counters[kCounterBound], 17);
            continue;
        }
        const DriverState<NC> &st = states[i];
        s.setup(pointFluid(F, a, i), st.sal);
        s.allocationSeedOutcome(a.P[i], a.T[i], st.z, k, memos[slot].seed[k]);
        evals += s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

// The role-permutation searches of the points the first recovery pass
// stopped: one warp per (point, permutation), each the nested flash under
// that permutation's roles (Solver::permutedFlash), written to the point's
// memo for the second pass.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedPermKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a)
{
    if (stagedTripped(a))
        return;
    const int queued = a.counters[kCounterPerm];
    const int64_t count = queued < a.allocCap ? queued : a.allocCap;
    const int lane = threadIdx.x & 31;
    const int64_t warpId = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    PermMemo<NC> *memos = static_cast<PermMemo<NC> *>(a.permMemos);
    const DriverState<NC> *states = static_cast<const DriverState<NC> *>(a.states);
    unsigned long long evals = 0;
    for (int64_t t = warpId; t < count * 6; t += nwarps)
    {
        const int slot = a.permSlots[t / 6];
        const int k = int(t % 6);
        int perm[3];
        swRolePermutation(k, perm);
        if (perm[0] == OIL && perm[1] == GAS && perm[2] == WATER)
            continue;   // the default roles: not part of the search
        if (slot < 0 || slot >= a.allocCap)
        {
            if (lane == 0)
                atomicExch(&a.counters[kCounterBound], 19);
            continue;
        }
        const int64_t i = a.allocPoints[slot];
        if (i < 0 || i >= a.n)
        {
            if (lane == 0)
                atomicExch(&a.counters[kCounterBound], 20);
            continue;
        }
        const DriverState<NC> &st = states[i];
        Solver<NC> s;
        s.setup(pointFluid(F, a, i), st.sal);
        s.lane = lane;
        s.width = 32;
        Result<NC> r;
        bool ok = false;
        double g = 0.0;
        s.permutedFlash(a.P[i], a.T[i], st.z, k, r, ok, g);
        __syncwarp();
        if (lane == 0)
        {
            PermOut<NC> &o = memos[slot].perm[k];
            o.r = r;
            o.gibbs = g;
            o.ok = ok ? 1 : 0;
            o.err = s.err;
            evals += s.evals;
        }
    }
    warpAddEvals(a.evalCounter, evals);
}

// Points whose main path did not end validated: the full solver with its
// fail-only recoveries, one warp per point.  The lanes run the point in
// lockstep and split the seeds of every stability test, which cuts the
// latency of these long recovery chains (they otherwise form the tail).
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedFullKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                 const __grid_constant__ nz_flash_out out, int phase)
{
    if (stagedTripped(a))
        return;
    const int count = a.counters[kCounterRest];
    const int lane = threadIdx.x & 31;
    const int warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long evals = 0;
    for (int k = warpId; k < count && k < a.n; k += nwarps)
    {
        const int64_t i = a.split[0][k];
        if (i < 0 || i >= a.n)
        {
            if (lane == 0)
                atomicExch(&a.counters[kCounterBound], 6);
            continue;
        }
        Solver<NC> s;
        s.setup(pointFluid(F, a, i), pointSalinity(F, a, i));
        s.lane = lane;
        s.width = 32;
        double zi[NC];
        for (int c = 0; c < NC; ++c)
            zi[c] = a.z[c * a.n + i];
        Result<NC> r;
        s.continuation = false;
        DriverState<NC> &ds = static_cast<DriverState<NC> *>(a.states)[i];
        // phase 0: one pass; phase 1: every point, those with memo slots
        // stopping where the role-permutation search starts; phase 2: the
        // stopped points, the search replayed from its memo
        const bool slotted = a.allocMemos && ds.allocSlot >= 0 && ds.allocSlot < a.allocCap;
        if (phase == 2 && !(ds.recoverFrom == 4 && slotted))
            continue;
        if (slotted && ds.recoverFrom == 3)
        {
            s.allocMemo = static_cast<const AllocMemo<NC> *>(a.allocMemos) + ds.allocSlot;
            s.stopAtPermutations = phase == 1 && a.permMemos != nullptr;
        }
        if (phase == 2)
            s.permMemo = static_cast<const PermMemo<NC> *>(a.permMemos) + ds.allocSlot;
        if (ds.recoverFrom > 0)
        {
            // the active-set path and the first recoveries already ran (and
            // failed) in the staged kernels: continue from that result
            r = ds.current;
            s.template recover<true>(a.P[i], a.T[i], ds.z, r, ds.recoverFrom);
        }
        else
            s.template flash<true>(a.P[i], a.T[i], zi, r);
        if (s.reachedPermutations)
        {
            // hand the point to the permutation kernel; phase 2 finishes it
            __syncwarp();
            if (lane == 0)
            {
                PermMemo<NC> &m = static_cast<PermMemo<NC> *>(a.permMemos)[ds.allocSlot];
                m.P = a.P[i];
                m.T = a.T[i];
                m.salinity = s.salinity;
                for (int c = 0; c < NC; ++c)
                    m.z[c] = ds.z[c];
                m.valid = 1;
                ds.recoverFrom = 4;
                const int q = atomicAdd(&a.counters[kCounterPerm], 1);
                if (q < a.allocCap)
                    a.permSlots[q] = ds.allocSlot;
                else
                    atomicExch(&a.counters[kCounterBound], 18);
                evals += s.evals;
            }
            continue;
        }
        if (s.err == ERR_NONE && !r.converged)
        {
            // Every recovery but the pressure continuation has failed.  Queue the
            // point for the anchor kernels (its failed result is written now and
            // replaced there if the continuation succeeds), or, with the queue
            // full, run the continuation here exactly as flash() would.
            int slot = 0;
            if (lane == 0)
                slot = atomicAdd(&a.counters[kCounterCont], 1);
            slot = __shfl_sync(0xffffffffu, slot, 0);
            if (slot < a.contCap)
            {
                if (lane == 0)
                {
                    a.cont[slot] = int(i);
                    evals += s.evals;
                    writeFlashOut<NC>(out, a.n, i, r, NZ_FLASH_FAILED);
                }
                continue;
            }
            double zn[NC];
            for (int c = 0; c < NC; ++c)
                zn[c] = zi[c];
            s.normalize(zn);
            Result<NC> continued;
            s.pressureContinuation(a.P[i], a.T[i], zn, continued);
            s.acceptContinued(a.P[i], a.T[i], zn, continued, r);
        }
        if (lane == 0)
        {
            evals += s.evals;
            const uint8_t status = s.err != ERR_NONE ? uint8_t(s.err)
                                                     : (r.converged ? uint8_t(NZ_FLASH_CONVERGED)
                                                                    : uint8_t(NZ_FLASH_FAILED));
            if (status != NZ_FLASH_CONVERGED && status != NZ_FLASH_FAILED)
                r.init();
            writeFlashOut<NC>(out, a.n, i, r, status);
        }
    }
    warpAddEvals(a.evalCounter, evals);
}

// Pressure-continuation anchors as each queued point's own chain: one warp per
// point runs its anchors in the fallback's order and stops at the first one
// with an outcome (the lanes splitting the stability seeds as in the recovery
// kernel) -- the fallback's own work, and no point waits for another's
// anchor before starting its next.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedAnchorChainKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a)
{
    if (stagedTripped(a))
        return;
    const int queued = a.counters[kCounterCont];
    const int64_t count = queued < a.contCap ? queued : a.contCap;
    const int lane = threadIdx.x & 31;
    const int64_t warpId = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    AnchorOut<NC> *anchors = static_cast<AnchorOut<NC> *>(a.anchors);
    unsigned long long evals = 0;
    for (int64_t k = warpId; k < count; k += nwarps)
    {
        const int64_t i = a.cont[k];
        if (i < 0 || i >= a.n)
        {
            if (lane == 0)
                atomicExch(&a.counters[kCounterBound], 8);
            continue;
        }
        double zn[NC];
#pragma unroll 1
        for (int an = 0; an < kAnchors; ++an)
        {
            Solver<NC> s;
            s.setup(pointFluid(F, a, i), pointSalinity(F, a, i));
            s.lane = lane;
            s.width = 32;
            for (int c = 0; c < NC; ++c)
                zn[c] = a.z[c * a.n + i];
            s.normalize(zn);
            Result<NC> r;
            const int outcome = s.continuationAnchor(a.P[i], a.T[i], zn, an, r);
            __syncwarp();
            if (lane == 0)
            {
                AnchorOut<NC> &o = anchors[k * kAnchors + an];
                o.outcome = outcome;
                o.err = s.err;
                if (outcome == CONT_SUCCESS)
                    o.r = r;
                evals += s.evals;
            }
            if (outcome != CONT_NONE)
                break;
        }
    }
    warpAddEvals(a.evalCounter, evals);
}

// The first anchor (in the fallback's order) with an outcome decides the point.
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedSelectKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                   const __grid_constant__ nz_flash_out out)
{
    if (stagedTripped(a))
        return;
    const int queued = a.counters[kCounterCont];
    const int64_t count = queued < a.contCap ? queued : a.contCap;
    const int lane = threadIdx.x & 31;
    const int64_t warpId = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const AnchorOut<NC> *anchors = static_cast<const AnchorOut<NC> *>(a.anchors);
    unsigned long long evals = 0;
    for (int64_t k = warpId; k < count; k += nwarps)
    {
        const int64_t i = a.cont[k];
        if (i < 0 || i >= a.n)
            continue;
        int chosen = -1;
        for (int an = 0; an < kAnchors; ++an)
            if (anchors[k * kAnchors + an].outcome != CONT_NONE)
            {
                chosen = an;
                break;
            }
        if (chosen < 0)
            continue;   // the failed result written by the recovery kernel stands
        const AnchorOut<NC> &o = anchors[k * kAnchors + chosen];
        if (o.outcome == CONT_ERROR)
        {
            if (lane == 0)
            {
                Result<NC> failed;
                failed.init();
                writeFlashOut<NC>(out, a.n, i, failed, uint8_t(o.err));
            }
            continue;
        }
        Solver<NC> s;
        s.setup(pointFluid(F, a, i), pointSalinity(F, a, i));
        s.lane = lane;
        s.width = 32;
        double zn[NC];
        for (int c = 0; c < NC; ++c)
            zn[c] = a.z[c * a.n + i];
        s.normalize(zn);
        Result<NC> continued = o.r;
        Result<NC> accepted;
        accepted.init();
        s.acceptContinued(a.P[i], a.T[i], zn, continued, accepted);
        if (lane == 0)
        {
            evals += s.evals;
            if (s.err != ERR_NONE)
            {
                accepted.init();
                writeFlashOut<NC>(out, a.n, i, accepted, uint8_t(s.err));
            }
            else if (accepted.converged)
                writeFlashOut<NC>(out, a.n, i, accepted, NZ_FLASH_CONVERGED);
        }
    }
    warpAddEvals(a.evalCounter, evals);
}

// The mixed-precision form's last step: the FP64 ln-fugacity Newton polish
// (Solver::polish) of every converged multiphase point, read back from and
// written to the output record (it needs at least the presence, status,
// fraction, composition and compressibility arrays; fields the caller left
// out stay out; the K-values are the flash's).
constexpr double kPolishTarget = 1.0e-11;   // largest ln-fugacity residual the polish aims for
constexpr int kPolishSteps = 4;

template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedPolishKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                   const __grid_constant__ nz_flash_out out)
{
    if (stagedTripped(a) || !out.status || !out.presence || !out.beta || !out.composition || !out.compressibility)
        return;
    unsigned long long evals = 0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n;
         i += int64_t(gridDim.x) * blockDim.x)
    {
        const uint8_t pres = out.presence[i];
        if (out.status[i] != NZ_FLASH_CONVERGED || popcount3(pres) < 2)
            continue;
        Solver<NC> s;
        s.setup(pointFluid(F, a, i), pointSalinity(F, a, i));
        double zn[NC];
        for (int c = 0; c < NC; ++c)
            zn[c] = a.z[c * a.n + i];
        s.normalize(zn);
        if (s.err)
            continue;
        Result<NC> r;
        r.init();
        r.converged = true;
        r.presence = pres;
        for (int p = 0; p < 3; ++p)
        {
            r.beta[p] = out.beta[p * a.n + i];
            r.Z[p] = out.compressibility[p * a.n + i];
            for (int c = 0; c < NC; ++c)
                r.x[p][c] = out.composition[(p * NC + c) * a.n + i];
        }
        const bool replaced = s.polish(a.P[i], a.T[i], zn, r, kPolishTarget, kPolishSteps);
        evals += s.evals;
        if (!replaced)
            continue;
        for (int p = 0; p < 3; ++p)
        {
            if (out.saturation) out.saturation[p * a.n + i] = r.sat[p];
            if (!(pres & bitOf(p)))
                continue;
            out.beta[p * a.n + i] = r.beta[p];
            for (int c = 0; c < NC; ++c)
                out.composition[(p * NC + c) * a.n + i] = r.x[p][c];
            if (out.compressibility) out.compressibility[p * a.n + i] = r.Z[p];
            if (out.molar_density) out.molar_density[p * a.n + i] = r.rho[p];
        }
    }
    warpAddEvals(a.evalCounter, evals);
}

template <int NC>
size_t stagedScratchBytes(int64_t n, const FluidDev &F)
{
    static_assert(sizeof(Rr3Memo<NC>) <= sizeof(TrialOut<NC>) * 3 * (NC + 6), "memo must fit a point's trial slots");
    const int nseeds = seedCount<NC>(F);
    size_t b = 0;
    auto add = [&](size_t bytes) { b += (bytes + 255) & ~size_t(255); };
    add(sizeof(DriverState<NC>) * size_t(n));
    add(sizeof(TrialOut<NC>) * size_t(n) * 3 * nseeds);
    add(sizeof(unsigned long long) * size_t(n) * 3);
    add(sizeof(unsigned long long) * size_t(n) * 3);
    add(sizeof(int) * size_t(n));
    add(sizeof(int) * size_t(n));
    add(sizeof(int) * size_t(n));
    add(sizeof(int) * size_t(n));
    add(sizeof(int) * size_t(n));
    add(sizeof(int) * kCounterWords);
    add(sizeof(unsigned long long) * size_t(n));
    add(sizeof(unsigned long long) * size_t(n));
    const int64_t cap = contCapacity(n);
    add(sizeof(int) * size_t(cap));
    add(sizeof(AnchorOut<NC>) * size_t(cap) * kAnchors);
    const int64_t acap = allocCapacity(n, F);
    if (acap > 0)
    {
        add(sizeof(AllocMemo<NC>) * size_t(acap));
        add(sizeof(int) * size_t(acap));
        add(sizeof(PermMemo<NC>) * size_t(acap));
        add(sizeof(int) * size_t(acap));
    }
    return b;
}

// Carve the scratch block into the staged buffers (same order as the size).
template <int NC>
StagedArgs stagedCarve(void *scratch, int64_t n, const FluidDev &F)
{
    const int nseeds = seedCount<NC>(F);
    StagedArgs a{};
    char *p = static_cast<char *>(scratch);
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~size_t(255);
        return r;
    };
    a.n = n;
    a.states = take(sizeof(DriverState<NC>) * size_t(n));
    a.trials = take(sizeof(TrialOut<NC>) * size_t(n) * 3 * nseeds);
    a.tasks[0] = reinterpret_cast<unsigned long long *>(take(sizeof(unsigned long long) * size_t(n) * 3));
    a.tasks[1] = reinterpret_cast<unsigned long long *>(take(sizeof(unsigned long long) * size_t(n) * 3));
    a.pending[0] = reinterpret_cast<int *>(take(sizeof(int) * size_t(n)));
    a.pending[1] = reinterpret_cast<int *>(take(sizeof(int) * size_t(n)));
    a.full = reinterpret_cast<int *>(take(sizeof(int) * size_t(n)));
    a.split[0] = reinterpret_cast<int *>(take(sizeof(int) * size_t(n)));
    a.split[1] = reinterpret_cast<int *>(take(sizeof(int) * size_t(n)));
    a.counters = reinterpret_cast<int *>(take(sizeof(int) * kCounterWords));
    a.threes = reinterpret_cast<unsigned long long *>(take(sizeof(unsigned long long) * size_t(n)));
    a.threesLong = reinterpret_cast<unsigned long long *>(take(sizeof(unsigned long long) * size_t(n)));
    a.contCap = contCapacity(n);
    a.cont = reinterpret_cast<int *>(take(sizeof(int) * size_t(a.contCap)));
    a.anchors = take(sizeof(AnchorOut<NC>) * size_t(a.contCap) * kAnchors);
    a.allocCap = allocCapacity(n, F);
    if (a.allocCap > 0)
    {
        a.allocMemos = take(sizeof(AllocMemo<NC>) * size_t(a.allocCap));
        a.allocPoints = reinterpret_cast<int *>(take(sizeof(int) * size_t(a.allocCap)));
        a.permMemos = take(sizeof(PermMemo<NC>) * size_t(a.allocCap));
        a.permSlots = reinterpret_cast<int *>(take(sizeof(int) * size_t(a.allocCap)));
    }
    return a;
}

// Launch shape of the staged kernels: resident blocks per SM of the lane
// kernels (TPD trials, three-phase step machine) and of the warp-per-point
// kernels.  The multi-model path picks them per component count by timing.
struct StagedTuning
{
    int laneBlocksPerSm = kTrialBlocksPerSm;
    int warpBlocksPerSm = 8;
};

// Launch sequence of one staged flash on `st`; the scratch block must hold
// stagedScratchBytes<NC>(n) bytes.  No allocation, no host synchronisation.
// `check` (null or two device ints) receives the batch's queue-bound and
// spin-guard codes (0 = none tripped).  The mixed form ends with the FP64
// ln-fugacity polish of its multiphase answers.
template <int NC>
int stagedLaunch(const FluidDev &F, void *scratch, int64_t n, const double *P, const double *T,
                 const double *z, const double *sal, const nz_flash_out &out,
                 unsigned long long *evalCounter, int smCount, cudaStream_t st, bool mixed = false,
                 int *check = nullptr, const StagedTuning &tune = StagedTuning(),
                 const FluidDev *fluids = nullptr, const uint16_t *model = nullptr)
{
    StagedArgs a = stagedCarve<NC>(scratch, n, F);
    a.mixed = mixed ? 1 : 0;
    a.fluids = fluids;
    a.model = model;
    const unsigned warpGrid = unsigned(smCount * tune.warpBlocksPerSm);
    a.P = P;
    a.T = T;
    a.z = z;
    a.sal = sal;
    a.evalCounter = evalCounter;
    cudaMemsetAsync(a.counters, 0, sizeof(int) * kCounterWords, st);
    const bool debugSync = stagedDebugSync();
    auto after = [&](const char *what, int round) {
        if (!debugSync)
            return 0;
        cudaError_t e = cudaStreamSynchronize(st);
        int c[kCounterWords];
        cudaMemcpy(c, a.counters, sizeof(c), cudaMemcpyDeviceToHost);
        const int r = round < kRoundSlots ? round : 0;
        fprintf(stderr, "[staged] %s round %d: %s tasks=%d pending=%d full=%d rest=%d cont=%d bound=%d guard=%d\n",
                what, round, cudaGetErrorString(e), c[4 * r], c[4 * r + 1], c[kCounterFull], c[kCounterRest],
                c[kCounterCont], c[kCounterBound], c[kCounterGuard]);
        return e == cudaSuccess && c[kCounterBound] == 0 && c[kCounterGuard] == 0 ? 0 : -1;
    };
    const unsigned gridN = unsigned((n + kFlashBlock - 1) / kFlashBlock);
    stagedStartKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out);
    if (after("start", 0))
        return setError(NZ_ERR_CUDA, "staged flash self-check failed after start");
    const unsigned trialGrid = unsigned(smCount * tune.laneBlocksPerSm);
    for (int round = 0; round + 1 < kMaxRounds; ++round)
    {
        if (mixed)
            stagedTrialMixedKernel<NC><<<trialGrid, kTrialBlock, 0, st>>>(F, a, round);
        stagedTrialKernel<NC><<<trialGrid, kTrialBlock, 0, st>>>(F, a, round);
        if (after("trial", round))
            return setError(NZ_ERR_CUDA, "staged flash self-check failed in trials");
        stagedClassifyKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, round);
        stagedResumeKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out, round, 0);
        stagedResumeKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out, round, 1);
        stagedThreeKernel<NC><<<trialGrid, kTrialBlock, 0, st>>>(F, a);
        stagedThreeLongKernel<NC><<<warpGrid, kFlashBlock, 0, st>>>(F, a);
        stagedThreeResumeKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out, round);
        stagedResetSplitKernel<<<1, 1, 0, st>>>(a.counters);
        if (after("resume", round + 1))
            return setError(NZ_ERR_CUDA, "staged flash self-check failed in resume");
    }
    stagedRr3MemoKernel<NC><<<warpGrid, kFlashBlock, 0, st>>>(F, a);
    stagedRecoverStartKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out);
    stagedThreeKernel<NC><<<trialGrid, kTrialBlock, 0, st>>>(F, a);
    stagedThreeLongKernel<NC><<<warpGrid, kFlashBlock, 0, st>>>(F, a);
    stagedRecoverThreeKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out);
    if (after("recover", kMaxRounds))
        return setError(NZ_ERR_CUDA, "staged flash self-check failed in recovery");
    for (int rr = 0; rr < kRecoveryRounds; ++rr)
    {
        if (mixed)
            stagedTrialMixedKernel<NC><<<trialGrid, kTrialBlock, 0, st>>>(F, a, kMaxRounds + rr);
        stagedTrialKernel<NC><<<trialGrid, kTrialBlock, 0, st>>>(F, a, kMaxRounds + rr);
        stagedRecoverResumeKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out, rr);
        if (after("recover round", kMaxRounds + rr + 1))
            return setError(NZ_ERR_CUDA, "staged flash self-check failed in recovery");
    }
    if (a.allocCap > 0)
    {
        stagedAllocQueueKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a);
        stagedAllocSeedKernel<NC><<<unsigned(smCount * tune.laneBlocksPerSm), kFlashBlock, 0, st>>>(F, a);
        stagedFullKernel<NC><<<warpGrid, kFlashBlock, 0, st>>>(F, a, out, 1);
        stagedPermKernel<NC><<<warpGrid, kFlashBlock, 0, st>>>(F, a);
        stagedFullKernel<NC><<<warpGrid, kFlashBlock, 0, st>>>(F, a, out, 2);
    }
    else
        stagedFullKernel<NC><<<warpGrid, kFlashBlock, 0, st>>>(F, a, out, 0);
    if (after("full", 0))
        return setError(NZ_ERR_CUDA, "staged flash self-check failed in the full solver");
    // each queued point's anchors as one warp's chain: the fallback's own
    // work, and the launch lasts as long as the longest chain
    stagedAnchorChainKernel<NC><<<warpGrid, kFlashBlock, 0, st>>>(F, a);
    stagedSelectKernel<NC><<<unsigned(smCount * 2), kFlashBlock, 0, st>>>(F, a, out);
    if (after("continuation", 0))
        return setError(NZ_ERR_CUDA, "staged flash self-check failed in the pressure continuation");
    if (mixed)
        stagedPolishKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out);
    stagedCheckKernel<<<1, 32, 0, st>>>(a.counters, check);
    return 0;
}

} // namespace nz
