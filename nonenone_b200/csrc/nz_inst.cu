// nz_inst.cu -- explicit instantiation of the per-component-count kernels.
// Compiled once per NZ_INST_NC value (3, 4, 5, 6, 8) so the heavy device code
// of each component count builds in its own translation unit.
#include "flash_kernels.cuh"
#include "staged_kernels.cuh"

#ifndef NZ_INST_NC
#error "NZ_INST_NC must be defined"
#endif

namespace nz
{
template int launchFlash<NZ_INST_NC>(nz_ctx *, int64_t, const double *, const double *, const double *,
                                     const double *, const nz_flash_out &, cudaStream_t);
template int launchEos<NZ_INST_NC>(nz_ctx *, int64_t, const double *, const double *, const double *,
                                   const int8_t *, const double *, double *, double *, cudaStream_t);
template int launchStability<NZ_INST_NC>(nz_ctx *, int64_t, const double *, const double *, const double *,
                                         const double *, const uint8_t *, const double *, uint8_t *,
                                         uint8_t *, uint8_t *, double *, double *, cudaStream_t);
template <int NC>
int launchStaged(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                 const double *sal, const nz_flash_out &out, bool mixed, cudaStream_t st)
{
    const size_t bytes = stagedScratchBytes<NC>(n, ctx->fluid);
    const int rc = ctx->ensureScratch(bytes);
    if (rc != 0)
        return rc;
    return stagedLaunch<NC>(ctx->fluid, ctx->scratch, n, P, T, z, sal, out, ctx->evalCounter, ctx->smCount, st,
                            mixed);
}
template <int NC>
int launchStagedInto(nz_ctx *ctx, void *scratch, size_t capacity, int64_t n, const double *P, const double *T,
                     const double *z, const double *sal, const nz_flash_out &out, bool mixed, cudaStream_t st)
{
    if (stagedScratchBytes<NC>(n, ctx->fluid) > capacity)
        return setError(NZ_ERR_ARGUMENT, "staged flash: work space too small");
    return stagedLaunch<NC>(ctx->fluid, scratch, n, P, T, z, sal, out, ctx->evalCounter, ctx->smCount, st,
                            mixed);
}
template <int NC>
size_t stagedScratchBytesNc(int64_t n, const FluidDev &F)
{
    return stagedScratchBytes<NC>(n, F);
}
template int launchStagedInto<NZ_INST_NC>(nz_ctx *, void *, size_t, int64_t, const double *, const double *,
                                          const double *, const double *, const nz_flash_out &, bool,
                                          cudaStream_t);
template size_t stagedScratchBytesNc<NZ_INST_NC>(int64_t, const FluidDev &);
template int launchStaged<NZ_INST_NC>(nz_ctx *, int64_t, const double *, const double *, const double *,
                                      const double *, const nz_flash_out &, bool, cudaStream_t);
} // namespace nz
