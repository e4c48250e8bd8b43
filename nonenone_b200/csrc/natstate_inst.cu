// natstate_inst.cu -- the Natural phase-state kernels (per-cell and staged
// update, P-T-z initialisation) of one component count, and the dispatch of
// every Natural operation (the assembly kernels live in natasm_inst.cu).
#include "natural_host.cuh"
#include "natural_kernels.cuh"
#include "natural_staged.cuh"

#ifndef NZ_INST_NC
#error "NZ_INST_NC must be defined"
#endif

namespace nz
{
template <int NC>
int natLaunchAssembly(int op, const NatLaunch &a, cudaStream_t st);

template <int NC>
int natLaunch(int op, const NatLaunch &a, cudaStream_t st)
{
    const int64_t n = a.g.ncell;
    // Phase-state solves: a warp per cell while the cells cannot fill the GPU
    // with threads, a thread per cell beyond that.
    int device = 0, smCount = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, device);
    const int width = n >= int64_t(smCount) * 256 ? 1 : 32;
    const unsigned warpGrid = unsigned((n * width + kNatBlock - 1) / kNatBlock);
    switch (op)
    {
    case NAT_CACHE:
    case NAT_RESIDUAL:
    case NAT_JACOBIAN:
    case NAT_HISTORY:
        return natLaunchAssembly<NC>(op, a, st);
    case NAT_UPDATE_PREPARE:
        return natStagedStability<NC>(a.F, a.K, n, a.primary, a.ps, a.stagedScratch, smCount, st);
    case NAT_UPDATE_REFLASH:
    {
        const NatStaged<NC> w = natStagedCarve<NC>(a.stagedScratch, n, a.F);
        return natReflash<NC>(a.F, n, a.stagedScratch, a.flashScratch, a.reflashCount, w.a.evalCounter, smCount,
                              st);
    }
    case NAT_UPDATE:
    {
        StabilityMemo<NC> *memo = nullptr;
        const FlashMemo<NC> *flashMemo = nullptr;
        if (a.stagedScratch)
        {
            const NatStaged<NC> w = natStagedCarve<NC>(a.stagedScratch, n, a.F);
            memo = w.memo;
            flashMemo = w.flash;
        }
        natUpdateKernel<NC><<<warpGrid, kNatBlock, 0, st>>>(a.F, a.K, n, a.primary, a.ps, a.newPrimary, a.newPs,
                                                           a.status, a.firstFailure, width, memo, flashMemo);
        if (stagedDebugSync())
        {
            const cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess)
                return cudaFail(e, "Natural update kernel");
        }
        break;
    }
    case NAT_INIT:
    {
        // with a work space: every cell's flash through the batched flash
        // first, the per-cell kernel then assigning from its memo
        FlashMemo<NC> *memos = nullptr;
        int initWidth = width;
        if (a.flashScratch)
        {
            const int rc = natInitFlash<NC>(a.F, a.K, n, a.initP, a.initZ, a.flashScratch, smCount, st, &memos);
            if (rc != NZ_OK)
                return rc;
            initWidth = 1;
        }
        const unsigned initGrid = unsigned((n * initWidth + kNatBlock - 1) / kNatBlock);
        natInitKernel<NC><<<initGrid, kNatBlock, 0, st>>>(a.F, a.K, n, a.initP, a.initZ, a.newPrimary, a.newPs,
                                                         a.firstFailure, initWidth, memos);
        break;
    }
    default:
        return setError(NZ_ERR_ARGUMENT, "natLaunch: unknown operation %d", op);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "Natural kernel launch");
}

template <int NC>
size_t natStagedBytesNc(int64_t n, const FluidDev &F)
{
    return natStagedBytes<NC>(n, F);
}

template <int NC>
size_t natReflashBytesNc(int64_t n, const FluidDev &F)
{
    return natReflashBytes<NC>(n, F);
}

template <int NC>
int *natReflashCountNc(void *scratch, int64_t n, const FluidDev &F)
{
    return natStagedCarve<NC>(scratch, n, F).count;
}

template <int NC>
size_t natInitBytesNc(int64_t n, const FluidDev &F)
{
    return natInitBytes<NC>(n, F);
}

template int natLaunch<NZ_INST_NC>(int, const NatLaunch &, cudaStream_t);
template size_t natInitBytesNc<NZ_INST_NC>(int64_t, const FluidDev &);
template size_t natStagedBytesNc<NZ_INST_NC>(int64_t, const FluidDev &);
template size_t natReflashBytesNc<NZ_INST_NC>(int64_t, const FluidDev &);
template int *natReflashCountNc<NZ_INST_NC>(void *, int64_t, const FluidDev &);
} // namespace nz
