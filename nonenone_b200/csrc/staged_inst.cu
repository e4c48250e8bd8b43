// staged_inst.cu -- the staged batched flash of one component count
// (NZ_INST_NC): its launch sequence and work-space sizes.
#include "staged_kernels.cuh"

#ifndef NZ_INST_NC
#error "NZ_INST_NC must be defined"
#endif

namespace nz
{
template <int NC>
int launchStaged(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                 const double *sal, const nz_flash_out &out, bool mixed, cudaStream_t st)
{
    const size_t bytes = stagedScratchBytes<NC>(n, ctx->fluid);
    const int rc = ctx->ensureScratch(bytes);
    if (rc != 0)
        return rc;
    return stagedLaunch<NC>(ctx->fluid, ctx->scratch, n, P, T, z, sal, out, ctx->evalCounter, ctx->smCount, st,
                            mixed, ctx->checkWords);
}
template <int NC>
int launchStagedInto(nz_ctx *ctx, void *scratch, size_t capacity, int64_t n, const double *P, const double *T,
                     const double *z, const double *sal, const nz_flash_out &out, bool mixed, cudaStream_t st)
{
    if (stagedScratchBytes<NC>(n, ctx->fluid) > capacity)
        return setError(NZ_ERR_ARGUMENT, "staged flash: work space too small");
    return stagedLaunch<NC>(ctx->fluid, scratch, n, P, T, z, sal, out, ctx->evalCounter, ctx->smCount, st,
                            mixed, ctx->checkWords);
}
template <int NC>
size_t stagedScratchBytesNc(int64_t n, const FluidDev &F)
{
    return stagedScratchBytes<NC>(n, F);
}
template <int NC>
int stagedLaunchExt(const FluidDev &F, void *scratch, int64_t n, const double *P, const double *T,
                    const double *z, const double *sal, const nz_flash_out &out,
                    unsigned long long *evalCounter, int smCount, cudaStream_t st, bool mixed)
{
    return stagedLaunch<NC>(F, scratch, n, P, T, z, sal, out, evalCounter, smCount, st, mixed);
}
// The staged launch sequence of a multi-model batch: per-point fluids from
// `fluids` (indexed by `model`), launch shape from the caller's tuning.
template <int NC>
int stagedLaunchModel(const FluidDev &F, void *scratch, int64_t n, const double *P, const double *T,
                      const double *z, const double *sal, const nz_flash_out &out,
                      unsigned long long *evalCounter, int smCount, cudaStream_t st, bool mixed, int *check,
                      int laneBlocksPerSm, int warpBlocksPerSm, const FluidDev *fluids, const uint16_t *model)
{
    StagedTuning tune;
    tune.laneBlocksPerSm = laneBlocksPerSm;
    tune.warpBlocksPerSm = warpBlocksPerSm;
    return stagedLaunch<NC>(F, scratch, n, P, T, z, sal, out, evalCounter, smCount, st, mixed, check, tune, fluids,
                            model);
}
template int stagedLaunchModel<NZ_INST_NC>(const FluidDev &, void *, int64_t, const double *, const double *,
                                           const double *, const double *, const nz_flash_out &,
                                           unsigned long long *, int, cudaStream_t, bool, int *, int, int,
                                           const FluidDev *, const uint16_t *);
template int stagedLaunchExt<NZ_INST_NC>(const FluidDev &, void *, int64_t, const double *, const double *,
                                         const double *, const double *, const nz_flash_out &,
                                         unsigned long long *, int, cudaStream_t, bool);
template int launchStagedInto<NZ_INST_NC>(nz_ctx *, void *, size_t, int64_t, const double *, const double *,
                                          const double *, const double *, const nz_flash_out &, bool,
                                          cudaStream_t);
template size_t stagedScratchBytesNc<NZ_INST_NC>(int64_t, const FluidDev &);
template int launchStaged<NZ_INST_NC>(nz_ctx *, int64_t, const double *, const double *, const double *,
                                      const double *, const nz_flash_out &, bool, cudaStream_t);
} // namespace nz
