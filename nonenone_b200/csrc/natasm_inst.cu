// natasm_inst.cu -- the Natural assembly kernels (frozen-exterior cache,
// residual, BAIJ Jacobian, history accumulation) of one component count.
#include "natural_host.cuh"
#include "natural_kernels.cuh"

#include <cstdlib>

#ifndef NZ_INST_NC
#error "NZ_INST_NC must be defined"
#endif

namespace nz
{
template <int NC, int KD>
int launchJacobianN(const NatLaunch &a, cudaStream_t st)
{
    using J = JacobianShape<NC, KD>;
    static bool attributeSet = false;
    if (!attributeSet)
    {
        const cudaError_t e = cudaFuncSetAttribute(natJacobianKernelN<NC, KD>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(J::smemBytes));
        if (e != cudaSuccess)
            return cudaFail(e, "Natural Jacobian shared memory");
        attributeSet = true;
    }
    const int64_t warps = (a.g.ncell + J::perWarp - 1) / J::perWarp;
    const unsigned grid = unsigned((warps * 32 + kNatBlock - 1) / kNatBlock);
    natJacobianKernelN<NC, KD><<<grid, kNatBlock, J::smemBytes, st>>>(a.F, a.K, a.g, a.primary, a.ps, a.values,
                                                                      a.residual, a.flag);
    return NZ_OK;
}

template <int NC>
int natLaunchAssembly(int op, const NatLaunch &a, cudaStream_t st)
{
    const int64_t n = a.g.ncell;
    const unsigned grid = unsigned((n + kNatBlock - 1) / kNatBlock);
    switch (op)
    {
    case NAT_CACHE:
        natCacheKernel<NC><<<grid, kNatBlock, 0, st>>>(a.F, a.K, a.g, a.primary, a.ps, a.flag);
        break;
    case NAT_RESIDUAL:
        natResidualKernel<NC><<<grid, kNatBlock, 0, st>>>(a.F, a.K, a.g, a.primary, a.ps, a.residual, a.flag);
        break;
    case NAT_JACOBIAN:
    {
        // directions per lane: 1 = natJacobianKernel, 2-5 natJacobianKernelN
        static const int kdir = [] {
            const char *v = std::getenv("NZ_JACOBIAN_K");
            return v ? std::atoi(v) : 5;
        }();
        if (kdir == 1)
        {
            constexpr int perWarp = 32 / Layout<NC>::B;
            const int64_t warps = (n + perWarp - 1) / perWarp;
            const unsigned jgrid = unsigned((warps * 32 + kNatBlock - 1) / kNatBlock);
            natJacobianKernel<NC><<<jgrid, kNatBlock, 0, st>>>(a.F, a.K, a.g, a.primary, a.ps, a.values,
                                                              a.residual, a.flag);
            break;
        }
        const int rc = kdir == 2   ? launchJacobianN<NC, 2>(a, st)
                       : kdir == 3 ? launchJacobianN<NC, 3>(a, st)
                       : kdir == 4 ? launchJacobianN<NC, 4>(a, st)
                                   : launchJacobianN<NC, 5>(a, st);
        if (rc != NZ_OK)
            return rc;
        break;
    }
    case NAT_HISTORY:
        natHistoryKernel<NC><<<grid, kNatBlock, 0, st>>>(a.F, a.K, a.g, a.primary, a.ps, a.prevAcc, a.flag);
        break;
    default:
        return setError(NZ_ERR_ARGUMENT, "natLaunchAssembly: unknown operation %d", op);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : cudaFail(e, "Natural kernel launch");
}

template int natLaunchAssembly<NZ_INST_NC>(int, const NatLaunch &, cudaStream_t);
} // namespace nz
