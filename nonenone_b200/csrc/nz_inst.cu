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
    (void)mixed;
    const size_t bytes = stagedScratchBytes<NC>(n, ctx->fluid);
    const int rc = ctx->ensureScratch(bytes);
    if (rc != 0)
        return rc;
    return stagedLaunch<NC>(ctx->fluid, ctx->scratch, n, P, T, z, sal, out, ctx->evalCounter, ctx->smCount, st);
}
template int launchStaged<NZ_INST_NC>(nz_ctx *, int64_t, const double *, const double *, const double *,
                                      const double *, const nz_flash_out &, bool, cudaStream_t);
} // namespace nz
