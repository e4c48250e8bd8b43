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
                              // [4*kMaxRounds]=full, +1 bound flag, +2 guard flag, +3 split1 of the current round
    unsigned long long *evalCounter;
};

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
    else if (stage == STAGE_NEED_FULL)
    {
        const int k = atomicAdd(&a.counters[4 * kMaxRounds], 1);
        if (k < a.n)
            a.full[k] = int(i);
        else
            atomicExch(&a.counters[4 * kMaxRounds + 1], 1);
    }
    else
    {
        const int q = round & 1;
        const int k = atomicAdd(&a.counters[4 * round + 1], 1);
        if (k < a.n && round < kMaxRounds)
            a.pending[q][k] = int(i);
        else
            atomicExch(&a.counters[4 * kMaxRounds + 1], 2);
        for (int cand = 0; cand < 3; ++cand)
            if (!(st.tested & bitOf(cand)))
            {
                const int t = atomicAdd(&a.counters[4 * round], 1);
                if (t < 3 * a.n)
                    a.tasks[q][t] = (static_cast<unsigned long long>(i) << 2) | unsigned(cand);
                else
                    atomicExch(&a.counters[4 * kMaxRounds + 1], 3);
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
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        Driver<NC> d;
        d.st = &states[i];
        const double sal = a.sal ? a.sal[i] : F.salinity;
        d.s.setup(&F, sal);
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
    const int q = round & 1;
    const int count = a.counters[4 * round + 1];
    const int nseeds = seedCount<NC>(F);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count && k < a.n; k += gridDim.x * blockDim.x)
    {
        const int64_t i = a.pending[q][k];
        if (i < 0 || i >= a.n)
        {
            atomicExch(&a.counters[4 * kMaxRounds + 1], 4);
            continue;
        }
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        const TrialOut<NC> *trials = static_cast<const TrialOut<NC> *>(a.trials) + i * 3 * nseeds;
        Driver<NC> d;
        d.st = &states[i];
        d.s.setup(&F, d.st->sal);
        d.combineStability(trials, nseeds, d.st->sr);
        bool adds = false;
        if (d.st->sr.valid && !d.st->sr.stable)
            for (int p = 0; p < 3; ++p)
                adds = adds || (!(d.st->tested & bitOf(p)) && d.st->sr.unstable[p]);
        const int which = adds ? 1 : 0;
        const int slot = atomicAdd(which ? &a.counters[4 * kMaxRounds + 3] : &a.counters[4 * round + 3], 1);
        if (slot < a.n)
            a.split[which][slot] = int(i);
        else
            atomicExch(&a.counters[4 * kMaxRounds + 1], 7);
    }
}

template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedResumeKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                   const __grid_constant__ nz_flash_out out, int round, int which)
{
    const int count = which ? a.counters[4 * kMaxRounds + 3] : a.counters[4 * round + 3];
    unsigned long long evals = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count && k < a.n; k += gridDim.x * blockDim.x)
    {
        const int64_t i = a.split[which][k];
        if (i < 0 || i >= a.n)
        {
            atomicExch(&a.counters[4 * kMaxRounds + 1], 4);
            continue;
        }
        DriverState<NC> *states = static_cast<DriverState<NC> *>(a.states);
        Driver<NC> d;
        d.st = &states[i];
        d.s.setup(&F, d.st->sal);
        const StabilityResult<NC> sr = d.st->sr;
        const uint8_t stage = d.activeSetLoop(true, &sr);
        routePoint<NC>(a, out, round + 1, i, stage, d);
        evals += d.s.evals;
    }
    warpAddEvals(a.evalCounter, evals);
}

// The split-1 counter is shared by the rounds; reset it between them.
static __global__ void stagedResetSplitKernel(int *counters) { counters[4 * kMaxRounds + 3] = 0; }

// Every (task, seed) TPD trial is a lane; idle lanes are refilled from the
// round's task list with one atomic per warp.
template <int NC>
__global__ void __launch_bounds__(kTrialBlock)
stagedTrialKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a, int round)
{
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
    const long long guardMax = 1LL << 26;
    while (true)
    {
        if (++guard > guardMax)
        {
            atomicExch(&a.counters[4 * kMaxRounds + 2], 1);
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
                        atomicExch(&a.counters[4 * kMaxRounds + 1], 5);
                    const DriverState<NC> &st = states[bad ? 0 : point];
                    evals += s.evals;
                    s.setup(&F, st.sal);
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
                    res.valid = 0;
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

// Points whose main path did not end validated: the full solver with its
// fail-only recoveries, one warp per point.  The lanes run the point in
// lockstep and split the seeds of every stability test, which cuts the
// latency of these long recovery chains (they otherwise form the tail).
template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stagedFullKernel(const __grid_constant__ FluidDev F, const __grid_constant__ StagedArgs a,
                 const __grid_constant__ nz_flash_out out)
{
    const int count = a.counters[4 * kMaxRounds];
    const int lane = threadIdx.x & 31;
    const int warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long evals = 0;
    for (int k = warpId; k < count && k < a.n; k += nwarps)
    {
        const int64_t i = a.full[k];
        if (i < 0 || i >= a.n)
        {
            if (lane == 0)
                atomicExch(&a.counters[4 * kMaxRounds + 1], 6);
            continue;
        }
        Solver<NC> s;
        s.setup(&F, a.sal ? a.sal[i] : F.salinity);
        s.lane = lane;
        s.width = 32;
        double zi[NC];
        for (int c = 0; c < NC; ++c)
            zi[c] = a.z[c * a.n + i];
        Result<NC> r;
        s.template flash<true>(a.P[i], a.T[i], zi, r);
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

template <int NC>
size_t stagedScratchBytes(int64_t n, const FluidDev &F)
{
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
    add(sizeof(int) * (4 * kMaxRounds + 4));
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
    a.counters = reinterpret_cast<int *>(take(sizeof(int) * (4 * kMaxRounds + 4)));
    return a;
}

// Launch sequence of one staged flash on `st`; the scratch block must hold
// stagedScratchBytes<NC>(n) bytes.  No allocation, no host synchronisation.
template <int NC>
int stagedLaunch(const FluidDev &F, void *scratch, int64_t n, const double *P, const double *T,
                 const double *z, const double *sal, const nz_flash_out &out,
                 unsigned long long *evalCounter, int smCount, cudaStream_t st)
{
    StagedArgs a = stagedCarve<NC>(scratch, n, F);
    a.P = P;
    a.T = T;
    a.z = z;
    a.sal = sal;
    a.evalCounter = evalCounter;
    cudaMemsetAsync(a.counters, 0, sizeof(int) * (4 * kMaxRounds + 4), st);
    const bool check = stagedDebugSync();
    auto after = [&](const char *what, int round) {
        if (!check)
            return 0;
        cudaError_t e = cudaStreamSynchronize(st);
        int c[4 * kMaxRounds + 4];
        cudaMemcpy(c, a.counters, sizeof(c), cudaMemcpyDeviceToHost);
        fprintf(stderr, "[staged] %s round %d: %s tasks=%d pending=%d full=%d bound=%d guard=%d\n", what, round,
                cudaGetErrorString(e), c[4 * (round < kMaxRounds ? round : 0)],
                c[4 * (round < kMaxRounds ? round : 0) + 1], c[4 * kMaxRounds], c[4 * kMaxRounds + 1],
                c[4 * kMaxRounds + 2]);
        return e == cudaSuccess && c[4 * kMaxRounds + 1] == 0 && c[4 * kMaxRounds + 2] == 0 ? 0 : -1;
    };
    const unsigned gridN = unsigned((n + kFlashBlock - 1) / kFlashBlock);
    stagedStartKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out);
    if (after("start", 0))
        return setError(NZ_ERR_CUDA, "staged flash self-check failed after start");
    const unsigned trialGrid = unsigned(smCount * kTrialBlocksPerSm);
    for (int round = 0; round + 1 < kMaxRounds; ++round)
    {
        stagedTrialKernel<NC><<<trialGrid, kTrialBlock, 0, st>>>(F, a, round);
        if (after("trial", round))
            return setError(NZ_ERR_CUDA, "staged flash self-check failed in trials");
        stagedClassifyKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, round);
        stagedResumeKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out, round, 0);
        stagedResumeKernel<NC><<<gridN, kFlashBlock, 0, st>>>(F, a, out, round, 1);
        stagedResetSplitKernel<<<1, 1, 0, st>>>(a.counters);
        if (after("resume", round + 1))
            return setError(NZ_ERR_CUDA, "staged flash self-check failed in resume");
    }
    stagedFullKernel<NC><<<unsigned(smCount * 8), kFlashBlock, 0, st>>>(F, a, out);
    if (after("full", 0))
        return setError(NZ_ERR_CUDA, "staged flash self-check failed in the full solver");
    return 0;
}

} // namespace nz
