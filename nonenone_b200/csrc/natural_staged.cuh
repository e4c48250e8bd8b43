// natural_staged.cuh -- the Natural phase-state update with its stability
// tests on the lane-per-trial kernel and its reflashes on the staged batched
// flash.
//
// updateStateWithReport (natural_petsc_runtime_state.inc:166-345) runs
// updatePhaseState on every cell.  A cell that keeps fewer than three phases
// runs a multi-seed TPD stability test (three_phase_equilibrium.hpp:467-487);
// a cell whose Newton saturation removed a phase first runs a restricted flash
// and tests its result (:398-463); an unstable or invalid test ends in a full
// P-T-z flash of the cell.  One thread per cell runs all of this at a few
// active lanes per warp.  Here the update takes four steps:
//
//   prefix    the head of every cell's update (decode, sanitize and the part
//             of updatePhaseState before any flash: Equilibrium::updateHead)
//             yields the input of the main-path test; cells that removed a
//             phase are listed and a second kernel runs their restricted flash
//             (the same Solver::flashRestricted on the same input) for the
//             input of theirs.  Each input is recorded in a StabilityMemo, the
//             test's reference-phase data prepared (Driver::prepareStability)
//             and one task per missing phase queued;
//   trials    stagedTrialKernel runs every (cell, missing phase, seed) trial
//             as its own lane; a combine kernel folds them in seed order
//             (Driver::combineStability) into the memo;
//   reflash   the cells whose answer calls for a full flash are listed and
//             flashed by the staged batched flash into per-cell FlashMemos;
//   update    the per-cell code runs from the start; its stability test and
//             its top-level flash find the memos with the identical input and
//             take the answers; anything else runs inline.
//
// The update computes every recorded input with the same functions on the same
// data, so the inputs match bit for bit; the combined test equals the
// sequential test and the staged flash equals flash() (the staged flash relies
// on the same equivalences).  An input that does not match simply runs inline.
#pragma once

#include "natural_kernels.cuh"
#include "staged_kernels.cuh"

namespace nz
{

// Work space of the staged update of n cells (carved by natStagedCarve).
template <int NC>
size_t natStagedBytes(int64_t n, const FluidDev &F)
{
    const int nseeds = seedCount<NC>(F);
    size_t b = 0;
    auto add = [&](size_t bytes) { b += (bytes + 255) & ~size_t(255); };
    add(sizeof(StabilityMemo<NC>) * size_t(n));
    add(sizeof(DriverState<NC>) * size_t(n));
    add(sizeof(TrialOut<NC>) * size_t(n) * 3 * nseeds);
    add(sizeof(unsigned long long) * size_t(n) * 3);
    add(sizeof(int) * kCounterWords);
    add(sizeof(unsigned long long));
    add(sizeof(FlashMemo<NC>) * size_t(n));
    add(size_t(n));                      // suppression flags after the update head
    add(sizeof(int64_t) * size_t(n));    // cells whose update reflashes
    add(sizeof(int));                    // their count
    add(sizeof(int64_t) * size_t(n));    // cells whose head removed a phase
    add(sizeof(int));                    // their count
    add(size_t(n));                      // path of each cell's recorded test
    return b;
}

// Which stability test a cell's memo holds, and what follows it in the update
// (three_phase_equilibrium.hpp:400-487).
constexpr uint8_t PATH_NONE = 0;      // nothing recorded: the update runs inline
constexpr uint8_t PATH_MAIN = 1;      // the main-path test of the active set
constexpr uint8_t PATH_REMOVED = 2;   // the test of the restricted flash's set after a phase removal
constexpr uint8_t PATH_REFLASH = 3;   // phase removed, restricted flash not converged: reflash directly

// The carved work space of the staged update.
template <int NC>
struct NatStaged
{
    StagedArgs a;
    StabilityMemo<NC> *memo;
    FlashMemo<NC> *flash;
    uint8_t *supp;
    int64_t *cells;
    int *count;
    int64_t *removed;
    int *removedCount;
    uint8_t *path;
};

template <int NC>
NatStaged<NC> natStagedCarve(void *scratch, int64_t n, const FluidDev &F)
{
    const int nseeds = seedCount<NC>(F);
    NatStaged<NC> w{};
    StagedArgs &a = w.a;
    char *p = static_cast<char *>(scratch);
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~size_t(255);
        return r;
    };
    a.n = n;
    w.memo = reinterpret_cast<StabilityMemo<NC> *>(take(sizeof(StabilityMemo<NC>) * size_t(n)));
    a.states = take(sizeof(DriverState<NC>) * size_t(n));
    a.trials = take(sizeof(TrialOut<NC>) * size_t(n) * 3 * nseeds);
    a.tasks[0] = reinterpret_cast<unsigned long long *>(take(sizeof(unsigned long long) * size_t(n) * 3));
    a.tasks[1] = a.tasks[0];   // only round 0 is used
    a.counters = reinterpret_cast<int *>(take(sizeof(int) * kCounterWords));
    a.evalCounter = reinterpret_cast<unsigned long long *>(take(sizeof(unsigned long long)));
    w.flash = reinterpret_cast<FlashMemo<NC> *>(take(sizeof(FlashMemo<NC>) * size_t(n)));
    w.supp = reinterpret_cast<uint8_t *>(take(size_t(n)));
    w.cells = reinterpret_cast<int64_t *>(take(sizeof(int64_t) * size_t(n)));
    w.count = reinterpret_cast<int *>(take(sizeof(int)));
    w.removed = reinterpret_cast<int64_t *>(take(sizeof(int64_t) * size_t(n)));
    w.removedCount = reinterpret_cast<int *>(take(sizeof(int)));
    w.path = reinterpret_cast<uint8_t *>(take(size_t(n)));
    return w;
}

// Record a cell's stability test (input, suppression flags, path), prepare its
// reference-phase data and queue one trial task per missing phase; a test
// that resolves without trials is stored as answered.
template <int NC>
__device__ void natRecordTest(const FluidDev &F, double T, int64_t ncell, const NatStaged<NC> &w, int64_t c, double P,
                              const double *z, uint8_t active, const double (&x)[3][NC], uint8_t suppression,
                              uint8_t path)
{
    const StagedArgs &a = w.a;
    StabilityMemo<NC> &m = w.memo[c];
    m.record(P, T, z, active, x);
    w.supp[c] = suppression;
    w.path[c] = path;
    DriverState<NC> &st = static_cast<DriverState<NC> *>(a.states)[c];
    st.P = P;
    st.T = T;
    st.sal = F.salinity;
    Driver<NC> d;
    d.s.setup(&F, F.salinity);
    d.st = &st;
    for (int i = 0; i < NC; ++i)
        st.z[i] = z[i];
    d.s.normalize(st.z);   // the seeds use the normalised feed, as stabilityTest does
    StabilityResult<NC> res;
    if (!d.prepareStability(P, T, z, active, x, res) || d.s.err != ERR_NONE)
    {
        m.res = res;
        m.err = d.s.err;
        m.state = MEMO_READY;
        return;
    }
    int missing = 0;
    for (int cand = 0; cand < 3; ++cand)
        if (!(active & bitOf(cand)))
            ++missing;
    int slot = atomicAdd(&a.counters[0], missing);
    if (slot < 0 || int64_t(slot) + missing > 3 * ncell)
    {
        atomicExch(&a.counters[kCounterBound], 21);   // self-check: the queue holds 3 tasks per cell
        return;
    }
    for (int cand = 0; cand < 3; ++cand)
        if (!(active & bitOf(cand)))
            a.tasks[0][slot++] = (static_cast<unsigned long long>(c) << 2) | unsigned(cand);
}

// Prefix pass: record each cell's main-path stability test and queue its trials.
template <int NC>
__global__ void __launch_bounds__(kNatBlock) natPrefixKernel(const __grid_constant__ FluidDev F,
                                                             const __grid_constant__ NatConst K, int64_t ncell,
                                                             const double *primary, const double *ps,
                                                             const __grid_constant__ NatStaged<NC> w)
{
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= ncell)
        return;
    const StagedArgs &a = w.a;
    StabilityMemo<NC> &m = w.memo[c];
    m.state = MEMO_NONE;
    m.err = ERR_NONE;
    w.flash[c].valid = 0;
    w.path[c] = PATH_NONE;
    UpdateHead<NC> h;
    if (!cellUpdateHead<NC>(F, K, primary, ps, c, h))
        return;
    if (h.removed)
    {
        const int k = atomicAdd(w.removedCount, 1);
        if (k >= 0 && k < ncell)
            w.removed[k] = c;
        return;
    }
    if (popcount3(h.active) == 3)
        return;
    natRecordTest<NC>(F, K.temperature, ncell, w, c, h.P, h.zt, h.active, h.comps, h.suppression, PATH_MAIN);
}

// Cells whose head removed a phase: their restricted flash (the same
// Solver::flashRestricted the update runs, on the same input) gives the set
// and compositions of the test that follows it.
template <int NC>
__global__ void __launch_bounds__(kNatBlock) natRemovedKernel(const __grid_constant__ FluidDev F,
                                                              const __grid_constant__ NatConst K, int64_t ncell,
                                                              const double *primary, const double *ps,
                                                              const __grid_constant__ NatStaged<NC> w)
{
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int listed = *w.removedCount;
    if (k >= listed || k >= ncell)
        return;
    const int64_t c = w.removed[k];
    if (c < 0 || c >= ncell)
        return;
    UpdateHead<NC> h;
    if (!cellUpdateHead<NC>(F, K, primary, ps, c, h))
        return;
    Solver<NC> s;
    s.setup(&F, F.salinity);
    Result<NC> reduced;
    s.flashRestricted(h.P, K.temperature, h.zt, h.active, &h.comps, reduced);
    if (s.err)
        return;   // the update fails this cell inline
    if (!reduced.converged)
    {
        StabilityMemo<NC> &m = w.memo[c];
        m.record(h.P, K.temperature, h.zt, 0, reduced.x);
        m.state = MEMO_NONE;   // no test: the flash input only
        w.path[c] = PATH_REFLASH;
        return;
    }
    if (popcount3(reduced.presence) == 3)
        return;
    natRecordTest<NC>(F, K.temperature, ncell, w, c, h.P, h.zt, reduced.presence, reduced.x, h.suppression,
                      PATH_REMOVED);
}

// Fold each cell's trials into its memo.  A trial kernel that tripped its
// bounds or guard check leaves the memos pending; the update then tests inline.
template <int NC>
__global__ void __launch_bounds__(kNatBlock) natCombineKernel(const __grid_constant__ FluidDev F, int64_t ncell,
                                                              const __grid_constant__ NatStaged<NC> w)
{
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= ncell)
        return;
    const StagedArgs &a = w.a;
    StabilityMemo<NC> &m = w.memo[c];
    if (m.state != MEMO_CAPTURED || a.counters[kCounterBound] != 0 || a.counters[kCounterGuard] != 0)
        return;
    const int nseeds = seedCount<NC>(F);
    Driver<NC> d;
    d.s.setup(&F, F.salinity);
    d.st = static_cast<DriverState<NC> *>(a.states) + c;
    StabilityResult<NC> res;
    d.combineStability(static_cast<const TrialOut<NC> *>(a.trials) + c * 3 * nseeds, nseeds, res);
    m.res = res;
    m.err = d.s.err;
    m.state = MEMO_READY;
}

// Cells whose main-path test found the missing phases unstable (or the test
// invalid) reflash the whole cell (three_phase_equilibrium.hpp:467-487):
// list them for the staged batched flash.
template <int NC>
__global__ void __launch_bounds__(kNatBlock) natSelectKernel(int64_t ncell, const __grid_constant__ NatStaged<NC> w)
{
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= ncell)
        return;
    const StabilityMemo<NC> &m = w.memo[c];
    const uint8_t path = w.path[c];
    if (path == PATH_NONE)
        return;
    if (path != PATH_REFLASH)
    {
        if (m.state != MEMO_READY || m.err != ERR_NONE)
            return;
        // main path: invalid or unstable; removed path: the same condition
        // (unstableMissing, :400-420)
        const bool invalid = !m.res.valid;
        if (!invalid && !Equilibrium<NC>::strongInstability(m.res, m.active, w.supp[c]))
            return;
    }
    const int k = atomicAdd(w.count, 1);
    if (k >= 0 && k < ncell)
        w.cells[k] = c;
}

// The listed cells' flash inputs (P, T, z component-major) for a batch of n.
template <int NC>
__global__ void natGatherKernel(int n, const __grid_constant__ NatStaged<NC> w, double *P, double *T, double *z)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const StabilityMemo<NC> &m = w.memo[w.cells[k]];
    P[k] = m.P;
    T[k] = m.T;
    for (int i = 0; i < NC; ++i)
        z[size_t(i) * n + k] = m.z[i];
}

// The batched flash's answers as per-cell flash memos (the Result that
// flash<true> returns, and its error code).
template <int NC>
__global__ void natScatterKernel(int n, const __grid_constant__ NatStaged<NC> w, const double *P, const double *T,
                                 const double *z, const __grid_constant__ nz_flash_out out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    FlashMemo<NC> &f = w.flash[w.cells[k]];
    f.P = P[k];
    f.T = T[k];
    for (int i = 0; i < NC; ++i)
        f.z[i] = z[size_t(i) * n + k];
    const uint8_t status = out.status[k];
    Result<NC> &r = f.r;
    r.converged = status == NZ_FLASH_CONVERGED;
    r.iterations = out.iterations[k];
    r.presence = out.presence[k];
    for (int p = 0; p < 3; ++p)
    {
        r.beta[p] = out.beta[size_t(p) * n + k];
        r.sat[p] = out.saturation[size_t(p) * n + k];
        r.Z[p] = out.compressibility[size_t(p) * n + k];
        r.rho[p] = out.molar_density[size_t(p) * n + k];
        for (int i = 0; i < NC; ++i)
            r.x[p][i] = out.composition[(size_t(p) * NC + i) * n + k];
    }
    for (int i = 0; i < NC; ++i)
    {
        r.Kg[i] = out.k_gas_oil[size_t(i) * n + k];
        r.Kw[i] = out.k_water_oil[size_t(i) * n + k];
    }
    f.err = status > NZ_FLASH_FAILED ? int(status) : ERR_NONE;
    f.valid = 1;
}

// Work space of the reflash batch of n cells: the staged flash's own, its
// inputs and its outputs.
template <int NC>
size_t natReflashBytes(int64_t n, const FluidDev &F)
{
    size_t b = stagedScratchBytes<NC>(n, F);
    auto add = [&](size_t bytes) { b += (bytes + 255) & ~size_t(255); };
    add(sizeof(double) * size_t(n) * (2 + NC));              // P, T, z
    add(size_t(n) * 2);                                       // status, presence
    add(sizeof(int32_t) * size_t(n));                         // iterations
    add(sizeof(double) * size_t(n) * (4 * 3 + 3 * NC + 2 * NC));
    return b;
}

// Gather, staged flash and scatter of the n listed cells on `st`.
template <int NC>
int natReflash(const FluidDev &F, int64_t ncell, void *scratch, void *flashScratch, int n, unsigned long long *evals,
               int smCount, cudaStream_t st)
{
    if (n <= 0)
        return NZ_OK;
    const NatStaged<NC> w = natStagedCarve<NC>(scratch, ncell, F);
    char *p = static_cast<char *>(flashScratch) + ((stagedScratchBytes<NC>(n, F) + 255) & ~size_t(255));
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~size_t(255);
        return r;
    };
    double *P = reinterpret_cast<double *>(take(sizeof(double) * size_t(n) * (2 + NC)));
    double *T = P + n;
    double *z = T + n;
    nz_flash_out out{};
    out.status = reinterpret_cast<uint8_t *>(take(size_t(n) * 2));
    out.presence = out.status + n;
    out.iterations = reinterpret_cast<int32_t *>(take(sizeof(int32_t) * size_t(n)));
    double *d = reinterpret_cast<double *>(take(sizeof(double) * size_t(n) * (4 * 3 + 3 * NC + 2 * NC)));
    out.beta = d;
    out.saturation = d + 3 * size_t(n);
    out.compressibility = d + 6 * size_t(n);
    out.molar_density = d + 9 * size_t(n);
    out.composition = d + 12 * size_t(n);
    out.k_gas_oil = out.composition + 3 * NC * size_t(n);
    out.k_water_oil = out.k_gas_oil + NC * size_t(n);
    const unsigned grid = unsigned((n + 255) / 256);
    natGatherKernel<NC><<<grid, 256, 0, st>>>(n, w, P, T, z);
    int rc = stagedLaunchExt<NC>(F, flashScratch, n, P, T, z, nullptr, out, evals, smCount, st, false);
    if (rc != 0)
        return rc;
    natScatterKernel<NC><<<grid, 256, 0, st>>>(n, w, P, T, z, out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "Natural reflash launch");
}

// P-T-z initialisation through the batched flash: every cell's input
// (P[c], the case temperature, z[c][:]) flashed by the staged kernels, the
// answers kept as per-cell flash memos for natInitKernel.
template <int NC>
size_t natInitBytes(int64_t n, const FluidDev &F)
{
    size_t b = 0;
    auto add = [&](size_t bytes) { b += (bytes + 255) & ~size_t(255); };
    add(stagedScratchBytes<NC>(n, F));
    add(sizeof(FlashMemo<NC>) * size_t(n));
    add(sizeof(double) * size_t(n) * (2 + NC));               // P, T, z
    add(size_t(n) * 2);                                        // status, presence
    add(sizeof(int32_t) * size_t(n));                          // iterations
    add(sizeof(double) * size_t(n) * (4 * 3 + 3 * NC + 2 * NC));
    add(sizeof(unsigned long long));                           // evaluation count
    return b;
}

template <int NC>
__global__ void natInitGatherKernel(int64_t n, const __grid_constant__ NatConst K, const double *Pin,
                                    const double *zin, double *P, double *T, double *z)
{
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < n; c += int64_t(gridDim.x) * blockDim.x)
    {
        P[c] = Pin[c];
        T[c] = K.temperature;
        for (int i = 0; i < NC; ++i)
            z[size_t(i) * n + c] = zin[c * NC + i];
    }
}

template <int NC>
__global__ void natInitMemoKernel(int64_t n, const __grid_constant__ NatConst K, const double *Pin,
                                  const double *zin, const __grid_constant__ nz_flash_out out, FlashMemo<NC> *memos)
{
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < n; c += int64_t(gridDim.x) * blockDim.x)
    {
        FlashMemo<NC> &f = memos[c];
        f.P = Pin[c];
        f.T = K.temperature;
        for (int i = 0; i < NC; ++i)
            f.z[i] = zin[c * NC + i];
        const uint8_t status = out.status[c];
        Result<NC> &r = f.r;
        r.converged = status == NZ_FLASH_CONVERGED;
        r.iterations = out.iterations[c];
        r.presence = out.presence[c];
        for (int p = 0; p < 3; ++p)
        {
            r.beta[p] = out.beta[size_t(p) * n + c];
            r.sat[p] = out.saturation[size_t(p) * n + c];
            r.Z[p] = out.compressibility[size_t(p) * n + c];
            r.rho[p] = out.molar_density[size_t(p) * n + c];
            for (int i = 0; i < NC; ++i)
                r.x[p][i] = out.composition[(size_t(p) * NC + i) * n + c];
        }
        for (int i = 0; i < NC; ++i)
        {
            r.Kg[i] = out.k_gas_oil[size_t(i) * n + c];
            r.Kw[i] = out.k_water_oil[size_t(i) * n + c];
        }
        f.err = status > NZ_FLASH_FAILED ? int(status) : ERR_NONE;
        f.valid = 1;
    }
}

// The batched flash of every cell into the memos carved from `scratch`
// (natInitBytes<NC>(n) bytes); returns the memos' address through `memos`.
template <int NC>
int natInitFlash(const FluidDev &F, const NatConst &K, int64_t n, const double *Pin, const double *zin,
                 void *scratch, int smCount, cudaStream_t st, FlashMemo<NC> **memos)
{
    char *p = static_cast<char *>(scratch);
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~size_t(255);
        return r;
    };
    void *flashScratch = take(stagedScratchBytes<NC>(n, F));
    FlashMemo<NC> *m = reinterpret_cast<FlashMemo<NC> *>(take(sizeof(FlashMemo<NC>) * size_t(n)));
    double *P = reinterpret_cast<double *>(take(sizeof(double) * size_t(n) * (2 + NC)));
    double *T = P + n;
    double *z = T + n;
    nz_flash_out out{};
    out.status = reinterpret_cast<uint8_t *>(take(size_t(n) * 2));
    out.presence = out.status + n;
    out.iterations = reinterpret_cast<int32_t *>(take(sizeof(int32_t) * size_t(n)));
    double *d = reinterpret_cast<double *>(take(sizeof(double) * size_t(n) * (4 * 3 + 3 * NC + 2 * NC)));
    out.beta = d;
    out.saturation = d + 3 * size_t(n);
    out.compressibility = d + 6 * size_t(n);
    out.molar_density = d + 9 * size_t(n);
    out.composition = d + 12 * size_t(n);
    out.k_gas_oil = out.composition + 3 * NC * size_t(n);
    out.k_water_oil = out.k_gas_oil + NC * size_t(n);
    unsigned long long *evals = reinterpret_cast<unsigned long long *>(take(sizeof(unsigned long long)));
    const int64_t blocks = (n + 255) / 256;
    const unsigned grid = unsigned(blocks < int64_t(smCount) * 8 ? blocks : int64_t(smCount) * 8);
    natInitGatherKernel<NC><<<grid, 256, 0, st>>>(n, K, Pin, zin, P, T, z);
    cudaMemsetAsync(evals, 0, sizeof(unsigned long long), st);
    int rc = stagedLaunchExt<NC>(F, flashScratch, n, P, T, z, nullptr, out, evals, smCount, st, false);
    if (rc != 0)
        return rc;
    natInitMemoKernel<NC><<<grid, 256, 0, st>>>(n, K, Pin, zin, out, m);
    *memos = m;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "Natural P-T-z initialisation flash");
}

// Prefix, trials, combine and select on `st`; afterwards the host reads the
// reflash count, runs natReflash, and the update kernel runs with the memos.
template <int NC>
int natStagedStability(const FluidDev &F, const NatConst &K, int64_t ncell, const double *primary,
                       const double *ps, void *scratch, int smCount, cudaStream_t st)
{
    const NatStaged<NC> w = natStagedCarve<NC>(scratch, ncell, F);
    const StagedArgs &a = w.a;
    cudaError_t e = cudaMemsetAsync(a.counters, 0, sizeof(int) * kCounterWords, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(a.evalCounter, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(w.count, 0, sizeof(int), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(w.removedCount, 0, sizeof(int), st);
    if (e != cudaSuccess)
        return cudaFail(e, "Natural staged update");
    // NZ_STAGED_SYNC=1: synchronise after every launch and name the one that failed
    const bool check = stagedDebugSync();
    auto after = [&](const char *what) {
        cudaError_t err = cudaGetLastError();
        if (err == cudaSuccess && check)
            err = cudaStreamSynchronize(st);
        if (err != cudaSuccess)
            return cudaFail(err, what);
        if (check)
        {
            int c[kCounterWords];
            cudaMemcpy(c, a.counters, sizeof(c), cudaMemcpyDeviceToHost);
            fprintf(stderr, "[natural staged] %s: tasks=%d bound=%d guard=%d\n", what, c[0], c[kCounterBound],
                    c[kCounterGuard]);
        }
        return int(NZ_OK);
    };
    const unsigned grid = unsigned((ncell + kNatBlock - 1) / kNatBlock);
    natPrefixKernel<NC><<<grid, kNatBlock, 0, st>>>(F, K, ncell, primary, ps, w);
    int rc = after("Natural staged update: prefix");
    if (rc != NZ_OK)
        return rc;
    natRemovedKernel<NC><<<grid, kNatBlock, 0, st>>>(F, K, ncell, primary, ps, w);
    if ((rc = after("Natural staged update: removed-phase cells")) != NZ_OK)
        return rc;
    stagedTrialKernel<NC><<<unsigned(smCount * kTrialBlocksPerSm), kTrialBlock, 0, st>>>(F, a, 0);
    if ((rc = after("Natural staged update: trials")) != NZ_OK)
        return rc;
    natCombineKernel<NC><<<grid, kNatBlock, 0, st>>>(F, ncell, w);
    if ((rc = after("Natural staged update: combine")) != NZ_OK)
        return rc;
    natSelectKernel<NC><<<grid, kNatBlock, 0, st>>>(ncell, w);
    return after("Natural staged update: select");
}

} // namespace nz
