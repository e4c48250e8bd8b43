// nz_flash.cu -- context management and the flash / EOS / stability entry
// points of the C ABI (include/nonenone_b200.h).
#include "common.cuh"

#include <cstdio>
#include <cstring>
#include <string>

namespace nz
{

thread_local std::string g_lastError;

int setError(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
    return code;
}

int cudaFail(cudaError_t e, const char *what)
{
    return setError(NZ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}


// Launchers, explicitly instantiated per NC in nz_inst.cu.
template <int NC>
int launchFlash(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                const double *sal, const nz_flash_out &out, cudaStream_t st);
template <int NC>
int launchEos(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *x,
              const int8_t *role, const double *sal, double *Z, double *lnphi, cudaStream_t st);
template <int NC>
int launchStability(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                    const double *sal, const uint8_t *active, const double *comps, uint8_t *stable,
                    uint8_t *valid, uint8_t *mask, double *ts, double *inc, cudaStream_t st);

} // namespace nz

using namespace nz;

extern "C" {

void nz_flash_options_default(nz_flash_options *o)
{
    if (!o)
        return;
    o->maximum_iterations = 120;
    o->maximum_rachford_rice_iterations = 80;
    o->maximum_stability_iterations = 80;
    o->stability_ssi_before_newton = 8;
    o->maximum_stability_newton = 12;
    o->two_phase_ssi_before_newton = 8;
    o->maximum_two_phase_newton = 12;
    o->three_phase_ssi_before_newton = 10;
    o->maximum_three_phase_newton = 12;
    o->fugacity_tolerance = 1.0e-9;
    o->rachford_rice_tolerance = 1.0e-12;
    o->stability_tolerance = 1.0e-9;
    o->phase_fraction_tolerance = 1.0e-10;
    o->coincident_composition_tolerance = 1.0e-8;
    o->composition_floor = 1.0e-30;
    o->log_k_step_limit = 2.0;
    o->numerical_jacobian_step = 1.0e-6;
}

const char *nz_last_error(void) { return g_lastError.c_str(); }

int32_t nz_abi_version(void) { return NZ_ABI_VERSION; }

int nz_ctx_create(const nz_fluid_desc *fluid, const nz_flash_options *options, int32_t device, nz_ctx **out)
{
    if (!fluid || !out)
        return setError(NZ_ERR_ARGUMENT, "nz_ctx_create: null argument");
    *out = nullptr;
    if (!ncSupported(fluid->nc))
        return setError(NZ_ERR_UNSUPPORTED, "nz_ctx_create: nc=%d not compiled (3,4,5,6,8)", fluid->nc);
    if (fluid->eos_model != NZ_EOS_PR && fluid->eos_model != NZ_EOS_SW && fluid->eos_model != NZ_EOS_CPA)
        return setError(NZ_ERR_UNSUPPORTED, "nz_ctx_create: unknown eos_model %d", fluid->eos_model);
    if (fluid->eos_model == NZ_EOS_CPA)
    {
        if (fluid->cpa_max_association_iterations <= 0 || !(fluid->cpa_association_tolerance > 0.0))
            return setError(NZ_ERR_ARGUMENT, "nz_ctx_create: CPA association iterations and tolerance must be positive");
        for (int i = 0; i < fluid->nc; ++i)
            if (!(fluid->cpa_b[i] > 0.0) || fluid->cpa_donor_sites[i] < 0 || fluid->cpa_acceptor_sites[i] < 0)
                return setError(NZ_ERR_ARGUMENT, "nz_ctx_create: CPA co-volume / site counts of component %d", i);
    }
    if (fluid->eos_type != 1 && fluid->eos_type != 5)
        return setError(NZ_ERR_ARGUMENT, "nz_ctx_create: eos_type must be 1 or 5");
    if (fluid->water_component < -1 || fluid->water_component >= fluid->nc)
        return setError(NZ_ERR_ARGUMENT, "nz_ctx_create: water_component out of range");
    if (fluid->eos_model == NZ_EOS_SW && fluid->water_component < 0)
        return setError(NZ_ERR_ARGUMENT, "nz_ctx_create: SW requires a water component");
    nz_flash_options opts;
    nz_flash_options_default(&opts);
    if (options)
        opts = *options;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess)
        return cudaFail(e, "cudaSetDevice");
    nz_ctx *c = new nz_ctx();
    c->device = device;
    c->desc = *fluid;
    c->options = opts;
    c->fluid = makeFluidDev(*fluid, opts);
    cudaDeviceGetAttribute(&c->smCount, cudaDevAttrMultiProcessorCount, device);
    // evaluation counter, then the two self-check words of the last batch
    e = cudaMalloc(&c->evalCounter, kCounterBlockBytes);
    if (e != cudaSuccess)
    {
        delete c;
        return cudaFail(e, "cudaMalloc(eval counter)");
    }
    c->checkWords = reinterpret_cast<int *>(c->evalCounter + 1);
    cudaMemset(c->evalCounter, 0, kCounterBlockBytes);
    *out = c;
    return NZ_OK;
}

int nz_ctx_destroy(nz_ctx *ctx)
{
    if (!ctx)
        return NZ_OK;
    cudaSetDevice(ctx->device);
    if (ctx->evalCounter)
        cudaFree(ctx->evalCounter);
    if (ctx->scratch)
        cudaFree(ctx->scratch);
    if (ctx->ownStream)
        cudaStreamDestroy(ctx->ownStream);
    delete ctx;
    return NZ_OK;
}

int nz_flash_eos_eval_count(nz_ctx *ctx, uint64_t *count)
{
    if (!ctx || !count)
        return setError(NZ_ERR_ARGUMENT, "nz_flash_eos_eval_count: null argument");
    unsigned long long v = 0;
    cudaError_t e = cudaMemcpy(&v, ctx->evalCounter, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_flash_eos_eval_count");
    *count = v;
    return NZ_OK;
}

int nz_eos_phase_batch(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *x,
                       const int8_t *role, const double *salinity, double *Z, double *lnphi, void *stream)
{
    if (!ctx || n < 0 || (n > 0 && (!P || !T || !x || !role || !Z || !lnphi)))
        return setError(NZ_ERR_ARGUMENT, "nz_eos_phase_batch: bad argument");
    if (n == 0)
        return NZ_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DISPATCH_NC(ctx->fluid.nc, launchEos, ctx, n, P, T, x, role, salinity, Z, lnphi, st);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "nz_eos_phase_batch launch");
}

int nz_flash_batch(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                   const double *salinity, const nz_flash_out *out, int32_t precision, void *stream)
{
    if (!ctx || !out || n < 0 || (n > 0 && (!P || !T || !z)))
        return setError(NZ_ERR_ARGUMENT, "nz_flash_batch: bad argument");
    if (precision != NZ_PRECISION_FP64 && precision != NZ_PRECISION_MIXED &&
        precision != NZ_PRECISION_FP64_STAGED)
        return setError(NZ_ERR_ARGUMENT, "nz_flash_batch: unknown precision %d", precision);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(ctx->evalCounter, 0, kCounterBlockBytes, st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_flash_batch counter reset");
    if (n == 0)
        return NZ_OK;
    if (precision == NZ_PRECISION_FP64)
    {
        DISPATCH_NC(ctx->fluid.nc, launchFlash, ctx, n, P, T, z, salinity, *out, st);
    }
    else
    {
        const bool mixed = precision == NZ_PRECISION_MIXED;
        DISPATCH_NC(ctx->fluid.nc, launchStaged, ctx, n, P, T, z, salinity, *out, mixed, st);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "nz_flash_batch launch");
}

int nz_stability_batch(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                       const double *salinity, const uint8_t *active, const double *comps, uint8_t *stable,
                       uint8_t *valid, uint8_t *mask, double *trialSum, double *incipient, void *stream)
{
    if (!ctx || n < 0 || (n > 0 && (!P || !T || !z || !active || !comps || !stable || !valid || !mask)))
        return setError(NZ_ERR_ARGUMENT, "nz_stability_batch: bad argument");
    if (n == 0)
        return NZ_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DISPATCH_NC(ctx->fluid.nc, launchStability, ctx, n, P, T, z, salinity, active, comps, stable, valid, mask,
                trialSum, incipient, st);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "nz_stability_batch launch");
}

int nz_flash_batch_host(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                        const double *salinity, const nz_flash_out *out, int32_t precision)
{
    if (!ctx || !out || n < 0)
        return setError(NZ_ERR_ARGUMENT, "nz_flash_batch_host: bad argument");
    if (n == 0)
        return NZ_OK;
    cudaSetDevice(ctx->device);
    const int nc = ctx->fluid.nc;
    const size_t nd = size_t(n) * sizeof(double);
    // input block P | T | z | sal, output block in nz_flash_out order
    const size_t inBytes = nd * (2 + nc + (salinity ? 1 : 0));
    const size_t outDoubles = size_t(n) * (3 * 4 + 3 * nc + 2 * nc);
    const size_t outBytes = outDoubles * sizeof(double) + size_t(n) * (2 + sizeof(int32_t));
    char *dev = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&dev), inBytes + outBytes + 256, ctx->hostStream());
    if (e != cudaSuccess)
        return cudaFail(e, "nz_flash_batch_host alloc");
    cudaStream_t st = ctx->hostStream();
    double *dP = reinterpret_cast<double *>(dev);
    double *dT = dP + n;
    double *dz = dT + n;
    double *ds = salinity ? dz + size_t(nc) * n : nullptr;
    cudaMemcpyAsync(dP, P, nd, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dT, T, nd, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dz, z, nd * nc, cudaMemcpyHostToDevice, st);
    if (ds)
        cudaMemcpyAsync(ds, salinity, nd, cudaMemcpyHostToDevice, st);
    double *o = reinterpret_cast<double *>(dev + inBytes);
    nz_flash_out dout{};
    dout.beta = o; o += 3 * n;
    dout.saturation = o; o += 3 * n;
    dout.compressibility = o; o += 3 * n;
    dout.molar_density = o; o += 3 * n;
    dout.composition = o; o += size_t(3) * nc * n;
    dout.k_gas_oil = o; o += size_t(nc) * n;
    dout.k_water_oil = o; o += size_t(nc) * n;
    dout.iterations = reinterpret_cast<int32_t *>(o);
    dout.presence = reinterpret_cast<uint8_t *>(dout.iterations + n);
    dout.status = dout.presence + n;
    int rc = nz_flash_batch(ctx, n, dP, dT, dz, ds, &dout, precision, st);
    if (rc == NZ_OK)
    {
        auto back = [&](void *h, const void *d, size_t bytes) {
            if (h)
                cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st);
        };
        back(out->beta, dout.beta, 3 * nd);
        back(out->saturation, dout.saturation, 3 * nd);
        back(out->compressibility, dout.compressibility, 3 * nd);
        back(out->molar_density, dout.molar_density, 3 * nd);
        back(out->composition, dout.composition, 3 * nc * nd);
        back(out->k_gas_oil, dout.k_gas_oil, nc * nd);
        back(out->k_water_oil, dout.k_water_oil, nc * nd);
        back(out->iterations, dout.iterations, size_t(n) * sizeof(int32_t));
        back(out->presence, dout.presence, size_t(n));
        back(out->status, dout.status, size_t(n));
    }
    cudaFreeAsync(dev, st);
    e = cudaStreamSynchronize(st);
    if (rc == NZ_OK && e != cudaSuccess)
        rc = cudaFail(e, "nz_flash_batch_host sync");
    if (rc == NZ_OK && precision != NZ_PRECISION_FP64)
    {
        int32_t bound = 0, guard = 0;
        rc = nz_flash_check(ctx, &bound, &guard);
        if (rc == NZ_OK && (bound || guard))
            rc = setError(NZ_ERR_SELFCHECK,
                          "nz_flash_batch_host: a device self-check stopped the batch (queue bound %d, spin guard %d); "
                          "points it left have status NZ_FLASH_UNFINISHED",
                          bound, guard);
    }
    return rc;
}

int nz_flash_check(nz_ctx *ctx, int32_t *bound_code, int32_t *guard_code)
{
    if (!ctx)
        return setError(NZ_ERR_ARGUMENT, "nz_flash_check: null context");
    int words[2] = {0, 0};
    cudaError_t e = cudaMemcpy(words, ctx->checkWords, sizeof(words), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_flash_check");
    if (bound_code)
        *bound_code = words[0];
    if (guard_code)
        *guard_code = words[1];
    return NZ_OK;
}

int nz_ctx_set_spin_limit(nz_ctx *ctx, int64_t limit)
{
    if (!ctx || limit < 1)
        return setError(NZ_ERR_ARGUMENT, "nz_ctx_set_spin_limit: need a context and a limit >= 1");
    ctx->fluid.spinLimit = limit;
    return NZ_OK;
}

} // extern "C"

namespace nz
{
size_t stagedScratchBytesFor(int nc, int64_t n, const FluidDev &F)
{
    switch (nc)
    {
    case 3: return stagedScratchBytesNc<3>(n, F);
    case 4: return stagedScratchBytesNc<4>(n, F);
    case 5: return stagedScratchBytesNc<5>(n, F);
    case 6: return stagedScratchBytesNc<6>(n, F);
    case 8: return stagedScratchBytesNc<8>(n, F);
    default: return ~size_t(0);
    }
}

int64_t stagedMaxPointsFor(int nc, size_t capacity, const FluidDev &F)
{
    int64_t lo = 0, hi = 1;
    while (stagedScratchBytesFor(nc, hi, F) <= capacity && hi < (int64_t(1) << 40))
        hi *= 2;
    while (hi - lo > 1)
    {
        const int64_t mid = (lo + hi) / 2;
        if (stagedScratchBytesFor(nc, mid, F) <= capacity)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}
} // namespace nz

int nz_ctx::ensureScratch(size_t bytes)
{
    if (bytes <= scratchBytes)
        return NZ_OK;
    if (scratch)
    {
        cudaFree(scratch);
        scratch = nullptr;
        scratchBytes = 0;
    }
    cudaError_t e = cudaMalloc(&scratch, bytes);
    if (e != cudaSuccess)
        return nz::cudaFail(e, "staged flash work space");
    scratchBytes = bytes;
    return NZ_OK;
}
