// nz_noalloc.cu -- the staged batched flash with its work space in a static
// device array, for callers that cannot allocate device memory at call time.
#include "common.cuh"

#include <mutex>

namespace
{
// Work space of nz_flash_batch_noalloc.  In host code this name is only a
// host-side stand-in; kernels get the device address from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char noallocScratch[NZ_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex setupMutex;
void *deviceAddress[kMaxDevices] = {};

// Once per device, with that device current: the array's device address.
int scratchAddress(int device, void **out)
{
    if (device < 0 || device >= kMaxDevices)
        return nz::setError(NZ_ERR_ARGUMENT, "nz_flash_batch_noalloc: device %d out of range", device);
    std::lock_guard<std::mutex> lock(setupMutex);
    if (deviceAddress[device] == nullptr)
    {
        int previous = 0;
        cudaError_t e = cudaGetDevice(&previous);
        if (e != cudaSuccess)
            return nz::cudaFail(e, "nz_flash_batch_noalloc cudaGetDevice");
        if (previous != device && (e = cudaSetDevice(device)) != cudaSuccess)
            return nz::cudaFail(e, "nz_flash_batch_noalloc cudaSetDevice");
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, noallocScratch);
        if (previous != device)
            cudaSetDevice(previous);
        if (e != cudaSuccess || ptr == nullptr)
            return nz::cudaFail(e, "nz_flash_batch_noalloc cudaGetSymbolAddress");
        deviceAddress[device] = ptr;
    }
    *out = deviceAddress[device];
    return NZ_OK;
}
} // namespace

extern "C" int nz_flash_batch_noalloc(nz_ctx *ctx, int64_t n, const double *P, const double *T,
                                      const double *z, const double *salinity, const nz_flash_out *out,
                                      int32_t precision, void *stream)
{
    using namespace nz;
    if (!ctx || !out || n < 0 || (n > 0 && (!P || !T || !z)))
        return setError(NZ_ERR_ARGUMENT, "nz_flash_batch_noalloc: bad argument");
    if (precision != NZ_PRECISION_FP64_STAGED && precision != NZ_PRECISION_MIXED)
        return setError(NZ_ERR_ARGUMENT,
                        "nz_flash_batch_noalloc: only the staged forms (FP64_STAGED, MIXED) are available");
    const size_t need = stagedScratchBytesFor(ctx->fluid.nc, n, ctx->fluid);
    if (need > NZ_NOALLOC_SCRATCH_BYTES)
        return setError(NZ_ERR_ARGUMENT,
                        "nz_flash_batch_noalloc: %lld points need %zu bytes of work space; the static "
                        "work space holds %llu bytes (at most %lld points for nc=%d)",
                        static_cast<long long>(n), need, NZ_NOALLOC_SCRATCH_BYTES,
                        static_cast<long long>(stagedMaxPointsFor(ctx->fluid.nc, NZ_NOALLOC_SCRATCH_BYTES,
                                                                  ctx->fluid)),
                        ctx->fluid.nc);
    void *scratch = nullptr;
    int rc = scratchAddress(ctx->device, &scratch);
    if (rc != NZ_OK)
        return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(ctx->evalCounter, 0, kCounterBlockBytes, st);
    if (e != cudaSuccess)
        return cudaFail(e, "nz_flash_batch_noalloc counter reset");
    if (n == 0)
        return NZ_OK;
    const bool mixed = precision == NZ_PRECISION_MIXED;
    DISPATCH_NC(ctx->fluid.nc, launchStagedInto, ctx, scratch, NZ_NOALLOC_SCRATCH_BYTES, n, P, T, z, salinity,
                *out, mixed, st);
    e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "nz_flash_batch_noalloc launch");
}
