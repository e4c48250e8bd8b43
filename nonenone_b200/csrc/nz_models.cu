// nz_models.cu -- uneven multi-model flash batches.
//
// Models (a fluid and its points each) are grouped by component count.  A
// group's points are gathered into one contiguous batch with a per-point
// model index; the staged flash runs on that batch with a device table of the
// group's fluids (every kernel reads the fluid of the point it holds), and the
// answers are scattered back into each model's own output arrays.  Groups run
// on forked streams; the whole call is captured once into a CUDA graph and
// replayed.  The autotuner times candidate launch shapes per component count
// on a strided sample of the group.
#include "common.cuh"

#include <algorithm>
#include <vector>

namespace nz
{
template <int NC>
int stagedLaunchModel(const FluidDev &F, void *scratch, int64_t n, const double *P, const double *T,
                      const double *z, const double *sal, const nz_flash_out &out,
                      unsigned long long *evalCounter, int smCount, cudaStream_t st, bool mixed, int *check,
                      int laneBlocksPerSm, int warpBlocksPerSm, const FluidDev *fluids, const uint16_t *model);

// The caller's arrays of one model, as the device kernels read them.
struct ModelPtrs
{
    const double *P;
    const double *T;
    const double *z;
    const double *sal;
    double salinity;   // used when sal is null
    int64_t n;
    nz_flash_out out;
};

namespace
{
constexpr int kModelsBlock = 256;

// Group batch point j_s (of `count`) <- point j = j_s * step of the group:
// model pmodel[j], its local index plocal[j].
__global__ void __launch_bounds__(kModelsBlock)
modelsGatherKernel(int64_t count, int64_t step, int nc, const uint16_t *pmodel, const int32_t *plocal,
                   const ModelPtrs *ptr, double *P, double *T, double *z, double *sal, uint16_t *model)
{
    for (int64_t js = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; js < count;
         js += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t j = js * step;
        const int m = pmodel[j];
        const int64_t l = plocal[j];
        const ModelPtrs &q = ptr[m];
        P[js] = q.P[l];
        T[js] = q.T[l];
        for (int c = 0; c < nc; ++c)
            z[c * count + js] = q.z[c * q.n + l];
        sal[js] = q.sal ? q.sal[l] : q.salinity;
        model[js] = uint16_t(m);
    }
}

// Group answers -> each model's outputs (fields the model left null are skipped).
__global__ void __launch_bounds__(kModelsBlock)
modelsScatterKernel(int64_t count, int nc, const uint16_t *pmodel, const int32_t *plocal, const ModelPtrs *ptr,
                    const __grid_constant__ nz_flash_out g)
{
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < count;
         j += int64_t(gridDim.x) * blockDim.x)
    {
        const ModelPtrs &q = ptr[pmodel[j]];
        const int64_t l = plocal[j];
        const int64_t n = q.n;
        const nz_flash_out &o = q.out;
        if (o.presence)
            o.presence[l] = g.presence[j];
        if (o.status)
            o.status[l] = g.status[j];
        if (o.iterations)
            o.iterations[l] = g.iterations[j];
        for (int p = 0; p < 3; ++p)
        {
            if (o.beta)
                o.beta[p * n + l] = g.beta[p * count + j];
            if (o.saturation)
                o.saturation[p * n + l] = g.saturation[p * count + j];
            if (o.compressibility)
                o.compressibility[p * n + l] = g.compressibility[p * count + j];
            if (o.molar_density)
                o.molar_density[p * n + l] = g.molar_density[p * count + j];
            if (o.composition)
                for (int c = 0; c < nc; ++c)
                    o.composition[(p * nc + c) * n + l] = g.composition[(p * nc + c) * count + j];
        }
        for (int c = 0; c < nc; ++c)
        {
            if (o.k_gas_oil)
                o.k_gas_oil[c * n + l] = g.k_gas_oil[c * count + j];
            if (o.k_water_oil)
                o.k_water_oil[c * n + l] = g.k_water_oil[c * count + j];
        }
    }
}

unsigned gridFor(int64_t count, int smCount)
{
    const int64_t blocks = (count + kModelsBlock - 1) / kModelsBlock;
    return unsigned(std::max<int64_t>(1, std::min<int64_t>(blocks, int64_t(smCount) * 16)));
}
} // namespace

// One component count's share of the models.
struct ModelGroup
{
    int nc{0};
    std::vector<int> members;   // model ids, in id order
    int tableOffset{0};         // first entry of this group in the pointer table
    int64_t points{0};
    FluidDev *fluids{nullptr};  // device [members]
    uint16_t *pmodel{nullptr};  // device [points]: local model index of each group point
    int32_t *plocal{nullptr};   // device [points]: index inside that model
    uint16_t *model{nullptr};   // device [points]: model index of each batch point (gathered)
    double *P{nullptr}, *T{nullptr}, *z{nullptr}, *sal{nullptr};
    nz_flash_out out{};
    void *outBlock{nullptr};
    void *scratch{nullptr};
    size_t scratchBytes{0};
    cudaStream_t stream{nullptr};
    cudaEvent_t done{nullptr};
    int laneBlocksPerSm{kTrialBlocksPerSm};
    int warpBlocksPerSm{8};
    // The fluid that sizes the group's work space and is passed as the
    // kernels' own fluid argument: the first member's, marked SW when any
    // member is SW (so the work space holds the SW allocation memos).  Every
    // point still reads its own model's fluid from the table.
    FluidDev shape{};
};
} // namespace nz

struct nz_models
{
    int device{0};
    int smCount{148};
    std::vector<nz::FluidDev> fluids;   // per model
    std::vector<int64_t> points;        // per model
    std::vector<nz::ModelGroup> groups;
    nz::ModelPtrs *hostTable{nullptr};  // pinned, group-major
    nz::ModelPtrs *devTable{nullptr};
    unsigned long long *evalCounter{nullptr};
    int *checks{nullptr};               // device [2 * groups]
    cudaStream_t stream{nullptr};       // capture stream
    cudaEvent_t fork{nullptr};
    cudaEvent_t lastLaunch{nullptr};
    bool launched{false};
    cudaGraphExec_t exec{nullptr};
    int graphPrecision{-1};

    void dropGraph()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        exec = nullptr;
        graphPrecision = -1;
    }
};

namespace nz
{
namespace
{
template <class T>
int devAlloc(T **p, size_t count, const char *what)
{
    *p = nullptr;
    if (count == 0)
        return NZ_OK;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T));
    return e == cudaSuccess ? NZ_OK : cudaFail(e, what);
}

void freeGroup(ModelGroup &g)
{
    for (void *p : {static_cast<void *>(g.fluids), static_cast<void *>(g.pmodel), static_cast<void *>(g.plocal),
                    static_cast<void *>(g.model), static_cast<void *>(g.P), static_cast<void *>(g.T),
                    static_cast<void *>(g.z), static_cast<void *>(g.sal), g.outBlock, g.scratch})
        if (p)
            cudaFree(p);
    if (g.stream)
        cudaStreamDestroy(g.stream);
    if (g.done)
        cudaEventDestroy(g.done);
    g = ModelGroup();
}

// The group's output arrays, carved from one block (the nz_flash_out layout
// for `points` points).
int allocGroupOutputs(ModelGroup &g)
{
    const int64_t n = g.points;
    const int nc = g.nc;
    const size_t doubles = size_t(n) * (4 * 3 + 3 * nc + 2 * nc);
    const size_t bytes = doubles * 8 + size_t(n) * (4 + 1 + 1) + 64;
    const cudaError_t e = cudaMalloc(&g.outBlock, bytes);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_models: group outputs");
    double *d = static_cast<double *>(g.outBlock);
    g.out.beta = d;
    d += 3 * n;
    g.out.saturation = d;
    d += 3 * n;
    g.out.compressibility = d;
    d += 3 * n;
    g.out.molar_density = d;
    d += 3 * n;
    g.out.composition = d;
    d += 3 * nc * n;
    g.out.k_gas_oil = d;
    d += nc * n;
    g.out.k_water_oil = d;
    d += nc * n;
    int32_t *it = reinterpret_cast<int32_t *>(d);
    g.out.iterations = it;
    uint8_t *u = reinterpret_cast<uint8_t *>(it + n);
    g.out.presence = u;
    g.out.status = u + n;
    return NZ_OK;
}

int launchGroup(const nz_models *m, int gi, int64_t count, bool mixed)
{
    const ModelGroup &g = m->groups[gi];
    const FluidDev &F = g.shape;
    nz_flash_out out = g.out;
    // the staged kernels address the outputs with the batch size as stride
    const int64_t n = count;
    out.beta = g.out.beta;
    out.saturation = g.out.beta + 3 * n;
    out.compressibility = g.out.beta + 6 * n;
    out.molar_density = g.out.beta + 9 * n;
    out.composition = g.out.beta + 12 * n;
    out.k_gas_oil = out.composition + 3 * g.nc * n;
    out.k_water_oil = out.k_gas_oil + g.nc * n;
    out.iterations = reinterpret_cast<int32_t *>(out.k_water_oil + g.nc * n);
    out.presence = reinterpret_cast<uint8_t *>(out.iterations + n);
    out.status = out.presence + n;
    int *check = m->checks + 2 * gi;
    const FluidDev *table = g.fluids;
    int rc = NZ_ERR_UNSUPPORTED;
    switch (g.nc)
    {
#define NZ_MODELS_CASE(NCV)                                                                                    \
    case NCV:                                                                                                  \
        rc = stagedLaunchModel<NCV>(F, g.scratch, n, g.P, g.T, g.z, g.sal, out, m->evalCounter, m->smCount,    \
                                    g.stream, mixed, check, g.laneBlocksPerSm, g.warpBlocksPerSm, table,       \
                                    g.model);                                                                  \
        break;
        NZ_MODELS_CASE(3)
        NZ_MODELS_CASE(4)
        NZ_MODELS_CASE(5)
        NZ_MODELS_CASE(6)
        NZ_MODELS_CASE(8)
#undef NZ_MODELS_CASE
    default:
        return setError(NZ_ERR_UNSUPPORTED, "nz_models: nc=%d not compiled", g.nc);
    }
    return rc;
}

// The group's whole sequence on its own stream: gather, staged flash, scatter.
int runGroup(const nz_models *m, int gi, bool mixed)
{
    const ModelGroup &g = m->groups[gi];
    const ModelPtrs *table = m->devTable + g.tableOffset;
    const unsigned grid = gridFor(g.points, m->smCount);
    modelsGatherKernel<<<grid, kModelsBlock, 0, g.stream>>>(g.points, 1, g.nc, g.pmodel, g.plocal, table, g.P, g.T,
                                                            g.z, g.sal, g.model);
    const int rc = launchGroup(m, gi, g.points, mixed);
    if (rc != 0)
        return rc;
    modelsScatterKernel<<<grid, kModelsBlock, 0, g.stream>>>(g.points, g.nc, g.pmodel, g.plocal, table, g.out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "nz_models: group launch");
}
} // namespace
} // namespace nz

using namespace nz;

extern "C" int nz_models_destroy(nz_models *m)
{
    if (!m)
        return NZ_OK;
    cudaSetDevice(m->device);
    if (m->launched && m->lastLaunch)
        cudaEventSynchronize(m->lastLaunch);
    m->dropGraph();
    for (ModelGroup &g : m->groups)
        freeGroup(g);
    if (m->hostTable)
        cudaFreeHost(m->hostTable);
    if (m->devTable)
        cudaFree(m->devTable);
    if (m->evalCounter)
        cudaFree(m->evalCounter);
    if (m->checks)
        cudaFree(m->checks);
    if (m->stream)
        cudaStreamDestroy(m->stream);
    if (m->fork)
        cudaEventDestroy(m->fork);
    if (m->lastLaunch)
        cudaEventDestroy(m->lastLaunch);
    delete m;
    return NZ_OK;
}

extern "C" int nz_models_create(int32_t nmodels, const nz_fluid_desc *fluids, const nz_flash_options *options,
                                const int64_t *points, int32_t device, nz_models **out)
{
    if (!fluids || !points || !out || nmodels <= 0)
        return setError(NZ_ERR_ARGUMENT, "nz_models_create: null argument or no models");
    *out = nullptr;
    if (nmodels > 65535)
        return setError(NZ_ERR_ARGUMENT, "nz_models_create: at most 65535 models");
    // validate every fluid exactly as a single-fluid context would
    for (int k = 0; k < nmodels; ++k)
    {
        nz_ctx *probe = nullptr;
        const int rc = nz_ctx_create(&fluids[k], options ? &options[k] : nullptr, device, &probe);
        if (rc != NZ_OK)
            return rc;
        nz_ctx_destroy(probe);
        if (points[k] < 0 || points[k] > INT32_MAX)
            return setError(NZ_ERR_ARGUMENT, "nz_models_create: model %d has %lld points", k, (long long)points[k]);
        if (fluids[k].water_component < 0)
            return setError(NZ_ERR_UNSUPPORTED, "nz_models_create: model %d has no water component "
                                                "(the models of a batch share the stability seed count)", k);
    }
    nz_models *m = new nz_models();
    m->device = device;
    cudaDeviceGetAttribute(&m->smCount, cudaDevAttrMultiProcessorCount, device);
    m->points.assign(points, points + nmodels);
    for (int k = 0; k < nmodels; ++k)
    {
        nz_flash_options o;
        nz_flash_options_default(&o);
        if (options)
            o = options[k];
        m->fluids.push_back(makeFluidDev(fluids[k], o));
    }
    auto fail = [&](int rc) {
        nz_models_destroy(m);
        return rc;
    };
    const int counts[5] = {3, 4, 5, 6, 8};
    int offset = 0;
    for (int nc : counts)
    {
        ModelGroup g;
        g.nc = nc;
        for (int k = 0; k < nmodels; ++k)
            if (fluids[k].nc == nc)
            {
                g.members.push_back(k);
                g.points += points[k];
            }
        if (g.members.empty() || g.points == 0)
            continue;
        if (g.points > (int64_t(1) << 28))
            return fail(setError(NZ_ERR_ARGUMENT, "nz_models_create: %lld points with nc=%d (at most 2^28 per "
                                                  "component count)", (long long)g.points, nc));
        g.tableOffset = offset;
        offset += int(g.members.size());
        m->groups.push_back(g);
        ModelGroup &G = m->groups.back();
        int rc = NZ_OK;
        rc = rc ? rc : devAlloc(&G.fluids, G.members.size(), "nz_models: fluid table");
        rc = rc ? rc : devAlloc(&G.pmodel, size_t(G.points), "nz_models: point models");
        rc = rc ? rc : devAlloc(&G.plocal, size_t(G.points), "nz_models: point indices");
        rc = rc ? rc : devAlloc(&G.model, size_t(G.points), "nz_models: batch models");
        rc = rc ? rc : devAlloc(&G.P, size_t(G.points), "nz_models: pressure");
        rc = rc ? rc : devAlloc(&G.T, size_t(G.points), "nz_models: temperature");
        rc = rc ? rc : devAlloc(&G.z, size_t(G.points) * nc, "nz_models: composition");
        rc = rc ? rc : devAlloc(&G.sal, size_t(G.points), "nz_models: salinity");
        rc = rc ? rc : allocGroupOutputs(G);
        if (rc)
            return fail(rc);
        G.shape = m->fluids[G.members[0]];
        for (int k : G.members)
            if (m->fluids[k].eosModel == NZ_EOS_SW)
                G.shape.eosModel = NZ_EOS_SW;
        G.scratchBytes = stagedScratchBytesFor(nc, G.points, G.shape);
        cudaError_t e = cudaMalloc(&G.scratch, G.scratchBytes);
        if (e != cudaSuccess)
            return fail(cudaFail(e, "nz_models: staged work space"));
        // the fluid table and the point -> (model, index) maps
        std::vector<FluidDev> table;
        std::vector<uint16_t> pm;
        std::vector<int32_t> pl;
        pm.reserve(size_t(G.points));
        pl.reserve(size_t(G.points));
        for (size_t t = 0; t < G.members.size(); ++t)
        {
            const int k = G.members[t];
            table.push_back(m->fluids[k]);
            for (int64_t l = 0; l < points[k]; ++l)
            {
                pm.push_back(uint16_t(t));
                pl.push_back(int32_t(l));
            }
        }
        e = cudaMemcpy(G.fluids, table.data(), table.size() * sizeof(FluidDev), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(G.pmodel, pm.data(), pm.size() * sizeof(uint16_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(G.plocal, pl.data(), pl.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&G.done, cudaEventDisableTiming);
        if (e != cudaSuccess)
            return fail(cudaFail(e, "nz_models: group set-up"));
    }
    cudaError_t e = cudaMallocHost(&m->hostTable, sizeof(ModelPtrs) * size_t(std::max(offset, 1)));
    if (e == cudaSuccess)
        e = cudaMalloc(&m->devTable, sizeof(ModelPtrs) * size_t(std::max(offset, 1)));
    if (e == cudaSuccess)
        e = cudaMalloc(&m->evalCounter, sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMalloc(&m->checks, sizeof(int) * 2 * std::max<size_t>(m->groups.size(), 1));
    if (e == cudaSuccess)
        e = cudaMemset(m->checks, 0, sizeof(int) * 2 * std::max<size_t>(m->groups.size(), 1));
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&m->fork, cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&m->lastLaunch, cudaEventDisableTiming);
    if (e != cudaSuccess)
        return fail(cudaFail(e, "nz_models: set-up"));
    *out = m;
    return NZ_OK;
}

namespace
{
bool stagedPrecision(int32_t precision)
{
    return precision == NZ_PRECISION_FP64_STAGED || precision == NZ_PRECISION_MIXED;
}

// Fill the pinned pointer table from the caller's arrays (group-major).
int fillTable(nz_models *m, const nz_model_io *io)
{
    if (m->launched)
    {
        // the previous replay may still be reading the table
        const cudaError_t e = cudaEventSynchronize(m->lastLaunch);
        if (e != cudaSuccess)
            return cudaFail(e, "nz_models: previous call");
    }
    for (const ModelGroup &g : m->groups)
        for (size_t t = 0; t < g.members.size(); ++t)
        {
            const int k = g.members[t];
            const nz_model_io &x = io[k];
            if (m->points[k] > 0 && (!x.pressure || !x.temperature || !x.z))
                return setError(NZ_ERR_ARGUMENT, "nz_models: model %d has null inputs", k);
            ModelPtrs &q = m->hostTable[g.tableOffset + int(t)];
            q.P = x.pressure;
            q.T = x.temperature;
            q.z = x.z;
            q.sal = x.salinity;
            q.salinity = m->fluids[k].salinity;
            q.n = m->points[k];
            q.out = x.out;
        }
    return NZ_OK;
}

size_t tableBytes(const nz_models *m)
{
    size_t entries = 0;
    for (const ModelGroup &g : m->groups)
        entries += g.members.size();
    return sizeof(ModelPtrs) * entries;
}

// Record the whole call on the capture stream: table upload, then every
// group on its own forked stream, joined at the end.
int captureGraph(nz_models *m, bool mixed)
{
    m->dropGraph();
    cudaStream_t st = m->stream;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_models: begin capture");
    int rc = NZ_OK;
    cudaMemsetAsync(m->evalCounter, 0, sizeof(unsigned long long), st);
    cudaMemcpyAsync(m->devTable, m->hostTable, tableBytes(m), cudaMemcpyHostToDevice, st);
    cudaEventRecord(m->fork, st);
    for (size_t gi = 0; gi < m->groups.size() && rc == NZ_OK; ++gi)
    {
        cudaStreamWaitEvent(m->groups[gi].stream, m->fork, 0);
        rc = runGroup(m, int(gi), mixed);
        cudaEventRecord(m->groups[gi].done, m->groups[gi].stream);
        cudaStreamWaitEvent(st, m->groups[gi].done, 0);
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(st, &graph);
    if (rc != NZ_OK)
    {
        if (graph)
            cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess)
        return cudaFail(e, "nz_models: end capture");
    e = cudaGraphInstantiate(&m->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess)
    {
        m->exec = nullptr;
        return cudaFail(e, "nz_models: graph instantiation");
    }
    m->graphPrecision = mixed ? NZ_PRECISION_MIXED : NZ_PRECISION_FP64_STAGED;
    return NZ_OK;
}

ModelGroup *groupOf(nz_models *m, int nc)
{
    for (ModelGroup &g : m->groups)
        if (g.nc == nc)
            return &g;
    return nullptr;
}
} // namespace

extern "C" int nz_models_flash(nz_models *m, const nz_model_io *io, int32_t precision, void *stream)
{
    if (!m || !io)
        return setError(NZ_ERR_ARGUMENT, "nz_models_flash: null argument");
    if (!stagedPrecision(precision))
        return setError(NZ_ERR_ARGUMENT, "nz_models_flash: precision must be FP64_STAGED or MIXED");
    cudaSetDevice(m->device);
    int rc = fillTable(m, io);
    if (rc)
        return rc;
    if (!m->exec || m->graphPrecision != precision)
    {
        rc = captureGraph(m, precision == NZ_PRECISION_MIXED);
        if (rc)
            return rc;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaGraphLaunch(m->exec, st);
    if (e == cudaSuccess)
        e = cudaEventRecord(m->lastLaunch, st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_models: graph launch");
    m->launched = true;
    return NZ_OK;
}

extern "C" int nz_models_tune(nz_models *m, const nz_model_io *io, int32_t precision, int64_t sample_points,
                              void *stream)
{
    if (!m || !io || sample_points <= 0)
        return setError(NZ_ERR_ARGUMENT, "nz_models_tune: bad argument");
    if (!stagedPrecision(precision))
        return setError(NZ_ERR_ARGUMENT, "nz_models_tune: precision must be FP64_STAGED or MIXED");
    cudaSetDevice(m->device);
    int rc = fillTable(m, io);
    if (rc)
        return rc;
    cudaStream_t caller = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaStreamSynchronize(caller);
    if (e == cudaSuccess)
        e = cudaMemcpy(m->devTable, m->hostTable, tableBytes(m), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_models_tune: set-up");
    const bool mixed = precision == NZ_PRECISION_MIXED;
    const size_t ng = m->groups.size();
    std::vector<cudaEvent_t> t0(ng), t1(ng);
    for (size_t g = 0; g < ng; ++g)
    {
        cudaEventCreate(&t0[g]);
        cudaEventCreate(&t1[g]);
    }
    std::vector<int64_t> count(ng);
    for (size_t gi = 0; gi < ng; ++gi)
    {
        ModelGroup &g = m->groups[gi];
        count[gi] = std::min(g.points, sample_points);
        const int64_t step = std::max<int64_t>(1, g.points / count[gi]);
        modelsGatherKernel<<<gridFor(count[gi], m->smCount), kModelsBlock, 0, g.stream>>>(
            count[gi], step, g.nc, g.pmodel, g.plocal, m->devTable + g.tableOffset, g.P, g.T, g.z, g.sal, g.model);
    }
    // One candidate shape per group, all groups at once on their own streams
    // (as they run in the graph); each group's time from its own events.
    auto timeAll = [&](const std::vector<int> &lane, const std::vector<int> &warp, std::vector<float> &ms) {
        for (size_t gi = 0; gi < ng; ++gi)
        {
            ModelGroup &g = m->groups[gi];
            g.laneBlocksPerSm = lane[gi];
            g.warpBlocksPerSm = warp[gi];
            cudaEventRecord(t0[gi], g.stream);
            const int r = launchGroup(m, int(gi), count[gi], mixed);
            cudaEventRecord(t1[gi], g.stream);
            if (r)
                return r;
        }
        for (size_t gi = 0; gi < ng; ++gi)
        {
            const cudaError_t se = cudaEventSynchronize(t1[gi]);
            if (se != cudaSuccess)
                return cudaFail(se, "nz_models_tune: sample run");
            cudaEventElapsedTime(&ms[gi], t0[gi], t1[gi]);
        }
        return int(NZ_OK);
    };
    // coordinate search: lane-kernel blocks at the default warp shape, then
    // warp-kernel blocks at each group's best lane shape (one untimed warm run)
    std::vector<int> lane(ng, kTrialBlocksPerSm), warp(ng, 8), bestLane(ng, kTrialBlocksPerSm), bestWarp(ng, 8);
    std::vector<float> ms(ng, 0.0f), best(ng, 0.0f);
    rc = timeAll(lane, warp, ms);
    bool first = true;
    for (int l : {2, 4, 8, 16})
    {
        if (rc)
            break;
        std::fill(lane.begin(), lane.end(), l);
        rc = timeAll(lane, warp, ms);
        for (size_t gi = 0; gi < ng && !rc; ++gi)
            if (first || ms[gi] < best[gi])
            {
                best[gi] = ms[gi];
                bestLane[gi] = l;
            }
        first = false;
    }
    for (int w : {4, 16})
    {
        if (rc)
            break;
        std::fill(warp.begin(), warp.end(), w);
        rc = timeAll(bestLane, warp, ms);
        for (size_t gi = 0; gi < ng && !rc; ++gi)
            if (ms[gi] < best[gi])
            {
                best[gi] = ms[gi];
                bestWarp[gi] = w;
            }
    }
    for (size_t gi = 0; gi < ng; ++gi)
    {
        m->groups[gi].laneBlocksPerSm = bestLane[gi];
        m->groups[gi].warpBlocksPerSm = bestWarp[gi];
        cudaEventDestroy(t0[gi]);
        cudaEventDestroy(t1[gi]);
    }
    m->dropGraph();
    return rc;
}

extern "C" int nz_models_get_tuning(nz_models *m, int32_t nc, int32_t *lane_blocks_per_sm,
                                    int32_t *warp_blocks_per_sm)
{
    if (!m || !lane_blocks_per_sm || !warp_blocks_per_sm)
        return setError(NZ_ERR_ARGUMENT, "nz_models_get_tuning: null argument");
    const ModelGroup *g = groupOf(m, nc);
    if (!g)
        return setError(NZ_ERR_ARGUMENT, "nz_models_get_tuning: no model with nc=%d", nc);
    *lane_blocks_per_sm = g->laneBlocksPerSm;
    *warp_blocks_per_sm = g->warpBlocksPerSm;
    return NZ_OK;
}

extern "C" int nz_models_set_tuning(nz_models *m, int32_t nc, int32_t lane_blocks_per_sm,
                                    int32_t warp_blocks_per_sm)
{
    if (!m)
        return setError(NZ_ERR_ARGUMENT, "nz_models_set_tuning: null argument");
    ModelGroup *g = groupOf(m, nc);
    if (!g)
        return setError(NZ_ERR_ARGUMENT, "nz_models_set_tuning: no model with nc=%d", nc);
    if (lane_blocks_per_sm < 1 || lane_blocks_per_sm > 64 || warp_blocks_per_sm < 1 || warp_blocks_per_sm > 64)
        return setError(NZ_ERR_ARGUMENT, "nz_models_set_tuning: blocks per SM must be in 1..64");
    g->laneBlocksPerSm = lane_blocks_per_sm;
    g->warpBlocksPerSm = warp_blocks_per_sm;
    m->dropGraph();
    return NZ_OK;
}

extern "C" int nz_models_check(nz_models *m, int32_t *bound_code, int32_t *guard_code)
{
    if (!m || !bound_code || !guard_code)
        return setError(NZ_ERR_ARGUMENT, "nz_models_check: null argument");
    cudaSetDevice(m->device);
    std::vector<int> c(2 * std::max<size_t>(m->groups.size(), 1), 0);
    const cudaError_t e = cudaMemcpy(c.data(), m->checks, sizeof(int) * c.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_models_check");
    int bound = 0, guard = 0;
    for (size_t g = 0; g < m->groups.size(); ++g)
    {
        bound = std::max(bound, c[2 * g]);
        guard = std::max(guard, c[2 * g + 1]);
    }
    *bound_code = bound;
    *guard_code = guard;
    return bound || guard ? NZ_ERR_SELFCHECK : NZ_OK;
}

extern "C" int nz_models_eos_eval_count(nz_models *m, uint64_t *count)
{
    if (!m || !count)
        return setError(NZ_ERR_ARGUMENT, "nz_models_eos_eval_count: null argument");
    cudaSetDevice(m->device);
    unsigned long long v = 0;
    const cudaError_t e = cudaMemcpy(&v, m->evalCounter, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_models_eos_eval_count");
    *count = v;
    return NZ_OK;
}
