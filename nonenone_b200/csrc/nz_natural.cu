// nz_natural.cu -- Natural assembly entry points: static topology, history,
// transactional phase-state update, residual and BAIJ Jacobian.
//
// Host-side restatement of the runtime shell around the kernels:
//   buildNaturalJacobianPattern (models/include/natural/petsc/jacobian_factory.hpp:39-245):
//     block rows = cells, columns = self + face neighbours, sorted; no wells
//   initializeStaticAssemblyCache_ (natural_petsc_runtime_cache_history.inc:8-146):
//     the block slot of every (cell, cell) and (neighbour, cell) pair
//   initializeLbcConstants_ (properties/compositional_properties.hpp:155-172)
//   updateStateWithReport (natural_petsc_runtime_state.inc:166-345): every cell
//     is updated into scratch; the first failing cell (lowest index) and its
//     flags form the report, and the scratch is committed only without failure.
#include "natural_host.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

// Selected names only: a namespace-wide using would put nz's double math
// overloads beside the CUDA headers' own.
using nz::cudaFail;
using nz::FluidDev;
using nz::kCentipoise;
using nz::kKelvinPerRankine;
using nz::kPsi;
using nz::NAT_CACHE;
using nz::NAT_HISTORY;
using nz::NAT_INIT;
using nz::NAT_JACOBIAN;
using nz::NAT_RESIDUAL;
using nz::NAT_UPDATE;
using nz::NAT_UPDATE_PREPARE;
using nz::NAT_UPDATE_REFLASH;
using nz::natLaunch;
using nz::natStagedBytesNc;
using nz::natReflashBytesNc;
using nz::natInitBytesNc;
using nz::natReflashCountNc;
using nz::NatConst;
using nz::NatGeom;
using nz::NatLaunch;
using nz::setError;

struct nz_natural
{
    nz_ctx *ctx{nullptr};
    int nc{0}, B{0}, NPS{0};
    int64_t ncell{0}, nconn{0}, nnzb{0};
    std::vector<int64_t> rowPtr, colIdx;
    NatConst K{};
    bool historySet{false};
    // device
    double *porosity{nullptr}, *volume{nullptr}, *trans{nullptr}, *gravity{nullptr};
    int64_t *offset{nullptr}, *neighbor{nullptr}, *selfSlot{nullptr}, *connSlot{nullptr};
    double *prevAcc{nullptr}, *cache{nullptr}, *newPrimary{nullptr}, *newPs{nullptr};
    uint8_t *status{nullptr};
    unsigned long long *firstFailure{nullptr};
    unsigned char *staged{nullptr};   // work space of the staged update (tests, memos, reflash list)
    int updateMode{NZ_UPDATE_AUTO};
    void *reflash{nullptr};           // work space of the update's batched reflash, grown on demand
    size_t reflashBytes{0};
    int *flag{nullptr};
    nz_report *report{nullptr};
    // pinned host mirror of flag / report
    struct Pinned
    {
        int flag;
        int reflashCount;
        nz_report report;
    } *pinned{nullptr};
    std::vector<void *> allocations;

    template <class T>
    int alloc(T *&p, size_t count)
    {
        void *v = nullptr;
        const cudaError_t e = cudaMalloc(&v, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess)
            return cudaFail(e, "nz_natural_create: cudaMalloc");
        allocations.push_back(v);
        p = static_cast<T *>(v);
        return NZ_OK;
    }
    template <class T>
    int upload(T *&p, const T *host, size_t count)
    {
        int rc = alloc(p, count);
        if (rc != NZ_OK)
            return rc;
        const cudaError_t e = cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice);
        return e == cudaSuccess ? NZ_OK : cudaFail(e, "nz_natural_create: upload");
    }

    NatGeom geom() const
    {
        NatGeom g{};
        g.ncell = ncell;
        g.porosity = porosity;
        g.volume = volume;
        g.offset = offset;
        g.neighbor = neighbor;
        g.trans = trans;
        g.gravity = gravity;
        g.selfSlot = selfSlot;
        g.connSlot = connSlot;
        g.prevAcc = prevAcc;
        g.cache = cache;
        return g;
    }

    NatLaunch launchArgs(const double *primary, const double *ps) const
    {
        NatLaunch a{};
        a.F = ctx->fluid;
        a.K = K;
        a.g = geom();
        a.primary = primary;
        a.ps = ps;
        a.flag = flag;
        return a;
    }

    ~nz_natural()
    {
        for (void *p : allocations)
            cudaFree(p);
        if (reflash)
            cudaFree(reflash);
        if (pinned)
            cudaFreeHost(pinned);
    }
};

namespace
{
size_t natStagedBytesFor(int nc, int64_t n, const FluidDev &F)
{
    switch (nc)
    {
    case 3: return natStagedBytesNc<3>(n, F);
    case 4: return natStagedBytesNc<4>(n, F);
    case 5: return natStagedBytesNc<5>(n, F);
    case 6: return natStagedBytesNc<6>(n, F);
    case 8: return natStagedBytesNc<8>(n, F);
    default: return 0;
    }
}

size_t natInitBytesFor(int nc, int64_t n, const FluidDev &F)
{
    switch (nc)
    {
    case 3: return natInitBytesNc<3>(n, F);
    case 4: return natInitBytesNc<4>(n, F);
    case 5: return natInitBytesNc<5>(n, F);
    case 6: return natInitBytesNc<6>(n, F);
    case 8: return natInitBytesNc<8>(n, F);
    default: return 0;
    }
}

size_t natReflashBytesFor(int nc, int64_t n, const FluidDev &F)
{
    switch (nc)
    {
    case 3: return natReflashBytesNc<3>(n, F);
    case 4: return natReflashBytesNc<4>(n, F);
    case 5: return natReflashBytesNc<5>(n, F);
    case 6: return natReflashBytesNc<6>(n, F);
    case 8: return natReflashBytesNc<8>(n, F);
    default: return 0;
    }
}

int *natReflashCountFor(int nc, void *scratch, int64_t n, const FluidDev &F)
{
    switch (nc)
    {
    case 3: return natReflashCountNc<3>(scratch, n, F);
    case 4: return natReflashCountNc<4>(scratch, n, F);
    case 5: return natReflashCountNc<5>(scratch, n, F);
    case 6: return natReflashCountNc<6>(scratch, n, F);
    case 8: return natReflashCountNc<8>(scratch, n, F);
    default: return nullptr;
    }
}

int natDispatch(int nc, int op, const NatLaunch &a, cudaStream_t st)
{
    switch (nc)
    {
    case 3: return natLaunch<3>(op, a, st);
    case 4: return natLaunch<4>(op, a, st);
    case 5: return natLaunch<5>(op, a, st);
    case 6: return natLaunch<6>(op, a, st);
    case 8: return natLaunch<8>(op, a, st);
    default: return setError(NZ_ERR_UNSUPPORTED, "nc=%d not compiled", nc);
    }
}

// The staged update's preparation: main-path stability tests on the trial
// kernels, then the batched flash of the cells that reflash.  Synchronises
// once, to size the reflash batch.
int natPrepareStagedUpdate(nz_natural *nat, NatLaunch &a, cudaStream_t st)
{
    a.stagedScratch = nat->staged;
    int rc = natDispatch(nat->nc, NAT_UPDATE_PREPARE, a, st);
    if (rc != NZ_OK)
        return rc;
    const FluidDev &F = nat->ctx->fluid;
    cudaError_t e = cudaMemcpyAsync(&nat->pinned->reflashCount, natReflashCountFor(nat->nc, nat->staged, nat->ncell, F),
                                    sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_update_state: reflash count");
    const int n = int(std::min<int64_t>(std::max(nat->pinned->reflashCount, 0), nat->ncell));
    if (n == 0)
        return NZ_OK;
    const size_t need = natReflashBytesFor(nat->nc, n, F);
    if (need > nat->reflashBytes)
    {
        if (nat->reflash)
            cudaFree(nat->reflash);
        nat->reflash = nullptr;
        nat->reflashBytes = 0;
        const size_t grow = need + need / 4;   // room for the next iterate's count
        e = cudaMalloc(&nat->reflash, grow);
        if (e != cudaSuccess)
            return cudaFail(e, "nz_update_state: reflash work space");
        nat->reflashBytes = grow;
    }
    a.flashScratch = nat->reflash;
    a.reflashCount = n;
    return natDispatch(nat->nc, NAT_UPDATE_REFLASH, a, st);
}

// Count the StableReducedSet cells before the first failure and fill the report.
__global__ void natReportKernel(int64_t ncell, const uint8_t *status, const unsigned long long *firstFailure,
                                nz_report *report)
{
    __shared__ unsigned long long partial[256];
    const unsigned long long first = *firstFailure;
    const int64_t limit = first < (unsigned long long)ncell ? int64_t(first) : ncell;
    unsigned long long reduced = 0;
    for (int64_t c = threadIdx.x; c < limit; c += blockDim.x)
        reduced += (status[c] & 3) == 1 ? 1ull : 0ull;
    partial[threadIdx.x] = reduced;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1)
    {
        if (int(threadIdx.x) < s)
            partial[threadIdx.x] += partial[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x != 0)
        return;
    nz_report r{};
    const bool failed = limit < ncell;
    r.succeeded = failed ? 0 : 1;
    r.first_failure_cell = failed ? limit : -1;
    r.updated_cells = limit;
    r.stable_reduced_cells = int64_t(partial[0]);
    r.failed_cells = failed ? 1 : 0;
    if (failed)
    {
        const uint8_t s = status[limit];
        r.status = s & 3;
        r.phase_removed = (s >> 2) & 1;
        r.missing_phase_unstable = (s >> 3) & 1;
        r.stability_invalid = (s >> 4) & 1;
        r.restricted_flash_failed = (s >> 5) & 1;
        r.unrestricted_flash_failed = (s >> 6) & 1;
    }
    *report = r;
}

// All-or-nothing commit of the updated primaries and phase states.
__global__ void natCommitKernel(int64_t ncell, int B, int NPS, const unsigned long long *firstFailure,
                                const double *newPrimary, const double *newPs, double *primary, double *ps)
{
    if (*firstFailure != ULLONG_MAX)
        return;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t np = ncell * B, ns = ncell * NPS;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < np; i += stride)
        primary[i] = newPrimary[i];
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < ns; i += stride)
        ps[i] = newPs[i];
}

int syncFlag(nz_natural *nat, cudaStream_t st, const char *what)
{
    cudaError_t e = cudaMemcpyAsync(&nat->pinned->flag, nat->flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return cudaFail(e, what);
    if (nat->pinned->flag)
        return setError(NZ_RECOVERABLE, "%s: a cell's thermodynamic evaluation failed (domain error)", what);
    return NZ_OK;
}

int validate(const nz_natural_desc &d, int64_t &nconn)
{
    if (d.ncell <= 0 || d.ncell > (int64_t(1) << 40))
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: ncell must be positive");
    if (!d.porosity || !d.volume || !d.conn_offset)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: null cell array");
    if (d.conn_offset[0] != 0)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: conn_offset[0] must be 0");
    for (int64_t c = 0; c < d.ncell; ++c)
        if (d.conn_offset[c + 1] < d.conn_offset[c])
            return setError(NZ_ERR_ARGUMENT, "nz_natural_create: conn_offset decreases at cell %lld", (long long)c);
    nconn = d.conn_offset[d.ncell];
    if (nconn > 0 && (!d.conn_neighbor || !d.conn_trans || !d.conn_gravity))
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: null connection array");
    if (!(d.time_step > 0.0) || !std::isfinite(d.time_step))
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: time_step must be positive");
    if (!(d.fugacity_scaling > 0.0) || !(d.temperature > 0.0))
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: fugacity_scaling and temperature must be positive");
    for (int64_t c = 0; c < d.ncell; ++c)
    {
        if (!(d.volume[c] > 0.0))
            return setError(NZ_ERR_ARGUMENT, "nz_natural_create: volume of cell %lld not positive", (long long)c);
        for (int64_t k = d.conn_offset[c]; k < d.conn_offset[c + 1]; ++k)
        {
            const int64_t nb = d.conn_neighbor[k];
            if (nb < 0 || nb >= d.ncell || nb == c)
                return setError(NZ_ERR_ARGUMENT, "nz_natural_create: bad neighbour %lld of cell %lld",
                                (long long)nb, (long long)c);
            // computeFaceMassFlux rejects these (face_flux.hpp:191-197)
            if (!(d.conn_trans[k] >= 0.0) || !std::isfinite(d.conn_trans[k]) || !std::isfinite(d.conn_gravity[k]))
                return setError(NZ_ERR_ARGUMENT, "nz_natural_create: connection %lld has a bad transmissibility",
                                (long long)k);
        }
    }
    return NZ_OK;
}
} // namespace

extern "C" {

int nz_natural_create(nz_ctx *ctx, const nz_natural_desc *desc, nz_natural **out)
{
    if (!out)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: null output");
    *out = nullptr;
    if (!ctx || !desc)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: null argument");
    if (ctx->fluid.eosModel == nz::EOS_CPA && ctx->fluid.cpa.symmetric < 0 && ctx->fluid.cpa.singleDonor < 0)
    {
        for (int i = 0; i < ctx->fluid.nc; ++i)
            if (ctx->fluid.cpa.donor[i] > 0)
                return setError(NZ_ERR_UNSUPPORTED,
                                "nz_natural_create: CPA with several donor-bearing components needs the general "
                                "association solve, which this build does not carry");
    }
    if (ctx->fluid.water < 0)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_create: the fully compositional model needs a water component");
    const nz_natural_desc &d = *desc;
    int64_t nconn = 0;
    int rc = validate(d, nconn);
    if (rc != NZ_OK)
        return rc;
    const int nc = ctx->fluid.nc;
    const int64_t n = d.ncell;

    // pattern: sorted self + neighbours; every connection must have its reverse
    std::vector<int64_t> rowPtr(n + 1, 0), colIdx;
    colIdx.reserve(size_t(n + nconn));
    for (int64_t c = 0; c < n; ++c)
    {
        const size_t begin = colIdx.size();
        colIdx.push_back(c);
        for (int64_t k = d.conn_offset[c]; k < d.conn_offset[c + 1]; ++k)
            colIdx.push_back(d.conn_neighbor[k]);
        std::sort(colIdx.begin() + begin, colIdx.end());
        if (std::adjacent_find(colIdx.begin() + begin, colIdx.end()) != colIdx.end())
            return setError(NZ_ERR_ARGUMENT, "nz_natural_create: cell %lld lists a neighbour twice", (long long)c);
        rowPtr[c + 1] = int64_t(colIdx.size());
    }
    auto slot = [&](int64_t row, int64_t col) -> int64_t {
        const auto b = colIdx.begin() + rowPtr[row], e = colIdx.begin() + rowPtr[row + 1];
        const auto it = std::lower_bound(b, e, col);
        return (it != e && *it == col) ? int64_t(it - colIdx.begin()) : -1;
    };
    std::vector<int64_t> selfSlot(n), connSlot(static_cast<size_t>(nconn));
    for (int64_t c = 0; c < n; ++c)
    {
        selfSlot[c] = slot(c, c);
        for (int64_t k = d.conn_offset[c]; k < d.conn_offset[c + 1]; ++k)
        {
            connSlot[k] = slot(d.conn_neighbor[k], c);
            if (connSlot[k] < 0)
                return setError(NZ_ERR_ARGUMENT, "nz_natural_create: connection %lld->%lld has no reverse",
                                (long long)c, (long long)d.conn_neighbor[k]);
        }
    }

    cudaSetDevice(ctx->device);
    nz_natural *nat = new nz_natural();
    nat->ctx = ctx;
    nat->nc = nc;
    nat->B = 3 * nc + 1;
    nat->NPS = 3 * nc + 8;
    nat->ncell = n;
    nat->nconn = nconn;
    nat->nnzb = rowPtr[n];
    nat->rowPtr = std::move(rowPtr);
    nat->colIdx = std::move(colIdx);

    NatConst &K = nat->K;
    K.temperature = d.temperature;
    K.timeStep = d.time_step;
    K.fugacityScaling = d.fugacity_scaling;
    K.swc = d.relperm.swc;
    K.sorw = d.relperm.sorw;
    K.sgc = d.relperm.sgc;
    K.sorg = d.relperm.sorg;
    K.krwMax = d.relperm.krw_max;
    K.krgMax = d.relperm.krg_max;
    K.kroMax = d.relperm.kro_max;
    for (int i = 0; i < nc; ++i)
    {
        const double mwSqrt = std::sqrt(1000.0 * ctx->desc.mw[i]);
        const double tcRankine = ctx->desc.tc[i] / kKelvinPerRankine;
        const double pcPsi = ctx->desc.pc[i] / kPsi;
        K.lbcMwSqrt[i] = mwSqrt;
        K.lbcEps[i] = 5.4402 * std::pow(tcRankine, 1.0 / 6.0) / (mwSqrt * std::pow(pcPsi, 2.0 / 3.0) * kCentipoise);
    }

    const int cacheFields = 10 + 3 * nc;
    if ((rc = nat->upload(nat->porosity, d.porosity, n)) || (rc = nat->upload(nat->volume, d.volume, n)) ||
        (rc = nat->upload(nat->offset, d.conn_offset, n + 1)) ||
        (rc = nat->upload(nat->neighbor, d.conn_neighbor, nconn)) ||
        (rc = nat->upload(nat->trans, d.conn_trans, nconn)) ||
        (rc = nat->upload(nat->gravity, d.conn_gravity, nconn)) ||
        (rc = nat->upload(nat->selfSlot, selfSlot.data(), n)) ||
        (rc = nat->upload(nat->connSlot, connSlot.data(), nconn)) || (rc = nat->alloc(nat->prevAcc, n * nc)) ||
        (rc = nat->alloc(nat->cache, n * cacheFields)) || (rc = nat->alloc(nat->newPrimary, n * nat->B)) ||
        (rc = nat->alloc(nat->newPs, n * nat->NPS)) || (rc = nat->alloc(nat->status, n)) ||
        (rc = nat->alloc(nat->firstFailure, 1)) || (rc = nat->alloc(nat->flag, 1)) ||
        (rc = nat->alloc(nat->report, 1)) ||
        (rc = nat->alloc(nat->staged, natStagedBytesFor(nc, n, ctx->fluid))))
    {
        delete nat;
        return rc;
    }
    cudaError_t e = cudaMallocHost(reinterpret_cast<void **>(&nat->pinned), sizeof(nz_natural::Pinned));
    if (e != cudaSuccess)
    {
        delete nat;
        return cudaFail(e, "nz_natural_create: pinned buffer");
    }
    *out = nat;
    return NZ_OK;
}

int nz_natural_destroy(nz_natural *nat)
{
    if (!nat)
        return NZ_OK;
    cudaSetDevice(nat->ctx->device);
    delete nat;
    return NZ_OK;
}

int nz_natural_set_update_mode(nz_natural *nat, int32_t mode)
{
    if (!nat)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_set_update_mode: null argument");
    if (mode != NZ_UPDATE_PER_CELL && mode != NZ_UPDATE_STAGED && mode != NZ_UPDATE_AUTO)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_set_update_mode: unknown mode %d", int(mode));
    nat->updateMode = mode;
    return NZ_OK;
}

int nz_natural_pattern(nz_natural *nat, int64_t *row_ptr, int64_t *col_idx, int64_t *nnzb)
{
    if (!nat)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_pattern: null handle");
    if (nnzb)
        *nnzb = nat->nnzb;
    if (row_ptr)
        std::copy(nat->rowPtr.begin(), nat->rowPtr.end(), row_ptr);
    if (col_idx)
        std::copy(nat->colIdx.begin(), nat->colIdx.end(), col_idx);
    return NZ_OK;
}

int nz_natural_init_ptz(nz_natural *nat, const double *P, const double *z, double *primary, double *phase_state,
                        int64_t *first_failure, void *stream)
{
    if (!nat || !P || !z || !primary || !phase_state)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_init_ptz: null argument");
    cudaSetDevice(nat->ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(nat->firstFailure, 0xff, sizeof(unsigned long long), st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_natural_init_ptz");
    NatLaunch a = nat->launchArgs(primary, phase_state);
    a.initP = P;
    a.initZ = z;
    a.newPrimary = nat->newPrimary;
    a.newPs = nat->newPs;
    a.firstFailure = nat->firstFailure;
    // every cell's flash through the batched flash (its work space held for
    // this call only), unless the per-cell update form was asked for
    void *initScratch = nullptr;
    if (nat->updateMode != NZ_UPDATE_PER_CELL)
    {
        e = cudaMalloc(&initScratch, natInitBytesFor(nat->nc, nat->ncell, nat->ctx->fluid));
        if (e != cudaSuccess)
            return cudaFail(e, "nz_natural_init_ptz: work space");
        a.flashScratch = initScratch;
    }
    int rc = natDispatch(nat->nc, NAT_INIT, a, st);
    if (rc != NZ_OK)
    {
        if (initScratch)
        {
            cudaStreamSynchronize(st);
            cudaFree(initScratch);
        }
        return rc;
    }
    const int64_t total = nat->ncell * std::max(nat->B, nat->NPS);
    const unsigned grid = unsigned(std::min<int64_t>((total + 255) / 256, 4 * 148));
    natCommitKernel<<<grid, 256, 0, st>>>(nat->ncell, nat->B, nat->NPS, nat->firstFailure, nat->newPrimary,
                                           nat->newPs, primary, phase_state);
    unsigned long long first = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&nat->pinned->report.first_failure_cell, nat->firstFailure, sizeof(first),
                            cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (initScratch)
        cudaFree(initScratch);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_natural_init_ptz");
    first = static_cast<unsigned long long>(nat->pinned->report.first_failure_cell);
    const bool failed = first != ULLONG_MAX;
    if (first_failure)
        *first_failure = failed ? int64_t(first) : -1;
    if (failed)
        return setError(NZ_RECOVERABLE, "nz_natural_init_ptz: P-T-z flash did not converge at cell %llu", first);
    return NZ_OK;
}

int nz_natural_set_history(nz_natural *nat, const double *primary, const double *phase_state, void *stream)
{
    if (!nat || !primary || !phase_state)
        return setError(NZ_ERR_ARGUMENT, "nz_natural_set_history: null argument");
    cudaSetDevice(nat->ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(nat->flag, 0, sizeof(int), st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_natural_set_history");
    NatLaunch a = nat->launchArgs(primary, phase_state);
    a.prevAcc = nat->prevAcc;
    int rc = natDispatch(nat->nc, NAT_HISTORY, a, st);
    if (rc != NZ_OK)
        return rc;
    rc = syncFlag(nat, st, "nz_natural_set_history");
    nat->historySet = rc == NZ_OK;
    return rc;
}

int nz_update_state(nz_natural *nat, double *primary, double *phase_state, nz_report *report, void *stream)
{
    if (!nat || !primary || !phase_state)
        return setError(NZ_ERR_ARGUMENT, "nz_update_state: null argument");
    cudaSetDevice(nat->ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(nat->firstFailure, 0xff, sizeof(unsigned long long), st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_update_state");
    NatLaunch a = nat->launchArgs(primary, phase_state);
    a.newPrimary = nat->newPrimary;
    a.newPs = nat->newPs;
    a.status = nat->status;
    a.firstFailure = nat->firstFailure;
    int rc = NZ_OK;
    bool staged = nat->updateMode == NZ_UPDATE_STAGED;
    if (nat->updateMode == NZ_UPDATE_AUTO)
    {
        int smCount = 148;
        cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, nat->ctx->device);
        staged = nat->ncell >= int64_t(smCount) * 256;
    }
    if (staged && (rc = natPrepareStagedUpdate(nat, a, st)) != NZ_OK)
        return rc;
    rc = natDispatch(nat->nc, NAT_UPDATE, a, st);
    if (rc != NZ_OK)
        return rc;
    natReportKernel<<<1, 256, 0, st>>>(nat->ncell, nat->status, nat->firstFailure, nat->report);
    const int64_t total = nat->ncell * std::max(nat->B, nat->NPS);
    const unsigned grid = unsigned(std::min<int64_t>((total + 255) / 256, 4 * 148));
    natCommitKernel<<<grid, 256, 0, st>>>(nat->ncell, nat->B, nat->NPS, nat->firstFailure, nat->newPrimary,
                                           nat->newPs, primary, phase_state);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&nat->pinned->report, nat->report, sizeof(nz_report), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_update_state");
    if (report)
        *report = nat->pinned->report;
    return nat->pinned->report.succeeded ? NZ_OK : NZ_RECOVERABLE;
}

int nz_residual(nz_natural *nat, const double *primary, const double *phase_state, double *residual, void *stream)
{
    if (!nat || !primary || !phase_state || !residual)
        return setError(NZ_ERR_ARGUMENT, "nz_residual: null argument");
    if (!nat->historySet)
        return setError(NZ_ERR_ARGUMENT, "nz_residual: call nz_natural_set_history first");
    cudaSetDevice(nat->ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(nat->flag, 0, sizeof(int), st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_residual");
    NatLaunch a = nat->launchArgs(primary, phase_state);
    a.residual = residual;
    int rc = natDispatch(nat->nc, NAT_CACHE, a, st);
    if (rc == NZ_OK)
        rc = natDispatch(nat->nc, NAT_RESIDUAL, a, st);
    if (rc != NZ_OK)
        return rc;
    return syncFlag(nat, st, "nz_residual");
}

static int jacobianInOrder(nz_natural *nat, const double *primary, const double *phase_state, double *values,
                           double *residual, void *stream, int columnOrder, const char *what)
{
    if (!nat || !primary || !phase_state || !values)
        return setError(NZ_ERR_ARGUMENT, "%s: null argument", what);
    if (!nat->historySet)
        return setError(NZ_ERR_ARGUMENT, "%s: call nz_natural_set_history first", what);
    cudaSetDevice(nat->ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(nat->flag, 0, sizeof(int), st);
    if (e != cudaSuccess)
        return cudaFail(e, what);
    NatLaunch a = nat->launchArgs(primary, phase_state);
    a.values = values;
    a.residual = residual;
    int rc = natDispatch(nat->nc, NAT_CACHE, a, st);
    a.g.columnOrder = columnOrder;
    if (rc == NZ_OK)
        rc = natDispatch(nat->nc, NAT_JACOBIAN, a, st);
    if (rc != NZ_OK)
        return rc;
    return syncFlag(nat, st, what);
}

int nz_jacobian(nz_natural *nat, const double *primary, const double *phase_state, double *baij_values,
                double *residual, void *stream)
{
    return jacobianInOrder(nat, primary, phase_state, baij_values, residual, stream, 0, "nz_jacobian");
}

int nz_jacobian_columns(nz_natural *nat, const double *primary, const double *phase_state, double *column_values,
                        double *residual, void *stream)
{
    return jacobianInOrder(nat, primary, phase_state, column_values, residual, stream, 1, "nz_jacobian_columns");
}

} // extern "C"
