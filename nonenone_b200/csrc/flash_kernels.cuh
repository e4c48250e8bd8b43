// flash_kernels.cuh -- flash / EOS / stability kernels and their launchers,
// instantiated once per component count by nz_inst.cu.
#pragma once

#include "common.cuh"
#include "flash.cuh"

namespace nz
{

// --------------------------------------------------------------- kernels --
__device__ __forceinline__ void addEvals(unsigned long long *counter, unsigned long long v)
{
    if (counter == nullptr)
        return;
    // one atomic per warp
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_down_sync(__activemask(), v, off);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(counter, v);
}

template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
flashKernel(const __grid_constant__ FluidDev F, int64_t n, const double *__restrict__ P,
            const double *__restrict__ T, const double *__restrict__ z,
            const double *__restrict__ salinity, const __grid_constant__ nz_flash_out out,
            unsigned long long *evalCounter)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    unsigned long long evals = 0;
    if (i < n)
    {
        Solver<NC> s;
        s.setup(&F, salinity ? salinity[i] : F.salinity);
        double zi[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c)
            zi[c] = z[c * n + i];
        Result<NC> r;
        s.template flash<true>(P[i], T[i], zi, r);
        evals = s.evals;
        const uint8_t status = s.err != ERR_NONE ? uint8_t(s.err)
                                                 : (r.converged ? uint8_t(NZ_FLASH_CONVERGED)
                                                                : uint8_t(NZ_FLASH_FAILED));
        if (status != NZ_FLASH_CONVERGED && status != NZ_FLASH_FAILED)
            r.init();
        if (out.status) out.status[i] = status;
        if (out.presence) out.presence[i] = r.converged && status == NZ_FLASH_CONVERGED ? r.presence : 0;
        if (out.iterations) out.iterations[i] = r.iterations;
#pragma unroll
        for (int p = 0; p < 3; ++p)
        {
            if (out.beta) out.beta[p * n + i] = r.beta[p];
            if (out.saturation) out.saturation[p * n + i] = r.sat[p];
            if (out.compressibility) out.compressibility[p * n + i] = r.Z[p];
            if (out.molar_density) out.molar_density[p * n + i] = r.rho[p];
            if (out.composition)
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    out.composition[(p * NC + c) * n + i] = r.x[p][c];
        }
#pragma unroll
        for (int c = 0; c < NC; ++c)
        {
            if (out.k_gas_oil) out.k_gas_oil[c * n + i] = r.Kg[c];
            if (out.k_water_oil) out.k_water_oil[c * n + i] = r.Kw[c];
        }
    }
    addEvals(evalCounter, evals);
}

template <int NC>
__global__ void __launch_bounds__(256)
eosKernel(const __grid_constant__ FluidDev F, int64_t n, const double *__restrict__ P,
          const double *__restrict__ T, const double *__restrict__ x, const int8_t *__restrict__ role,
          const double *__restrict__ salinity, double *__restrict__ Zout, double *__restrict__ lnphi)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int r = role[i];
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (F.eosModel == EOS_CPA)
    {
        double xc[NC], phi[NC], Z = 0.0;
        for (int c = 0; c < NC; ++c)
            xc[c] = x[c * n + i];
        const bool ok = cpaPhase<NC>(F, P[i], T[i], xc, r != GAS, Z, phi) == ERR_NONE;
        Zout[i] = ok ? Z : nan;
        for (int c = 0; c < NC; ++c)
            lnphi[c * n + i] = ok ? log(phi[c]) : nan;
        return;
    }
    MixParams<NC> p;
    mixingParameters<NC>(F, P[i], T[i], salinity ? salinity[i] : F.salinity, r == WATER, p);
    double xi[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c)
        xi[c] = x[c * n + i];
    PhaseMix<NC> m;
    phaseMixing<NC>(xi, p, m);
    const double Z = selectCubicRoot(m.A, m.B, F.m1, F.m2, r == GAS);
    double phi[NC];
    const bool ok = isfinite(Z) && fugacityCoefficients<NC>(xi, p, m, Z, F.m1, F.m2, phi);
    Zout[i] = ok ? Z : nan;
#pragma unroll
    for (int c = 0; c < NC; ++c)
        lnphi[c * n + i] = ok ? log(phi[c]) : nan;
}

template <int NC>
__global__ void __launch_bounds__(kFlashBlock)
stabilityKernel(const __grid_constant__ FluidDev F, int64_t n, const double *__restrict__ P,
                const double *__restrict__ T, const double *__restrict__ z,
                const double *__restrict__ salinity, const uint8_t *__restrict__ active,
                const double *__restrict__ comps, uint8_t *stable, uint8_t *valid,
                uint8_t *unstableMask, double *trialSum, double *incipient)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    Solver<NC> s;
    s.setup(&F, salinity ? salinity[i] : F.salinity);
    double zi[NC];
    double x[3][NC];
#pragma unroll
    for (int c = 0; c < NC; ++c)
        zi[c] = z[c * n + i];
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
        for (int c = 0; c < NC; ++c)
            x[p][c] = comps[(p * NC + c) * n + i];
    StabilityResult<NC> st;
    s.stabilityTest(P[i], T[i], zi, active[i], x, st);
    if (s.err)
    {
        stable[i] = 0;
        valid[i] = 0;
        unstableMask[i] = 0xff;
        return;
    }
    stable[i] = st.stable;
    valid[i] = st.valid;
    uint8_t m = 0;
#pragma unroll
    for (int p = 0; p < 3; ++p)
    {
        if (st.unstable[p]) m |= uint8_t(1u << p);
        if (trialSum) trialSum[p * n + i] = st.trialSum[p];
        if (incipient)
#pragma unroll
            for (int c = 0; c < NC; ++c)
                incipient[(p * NC + c) * n + i] = st.incipient[p][c];
    }
    unstableMask[i] = m;
}

template <int NC>
int launchFlash(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                const double *sal, const nz_flash_out &out, cudaStream_t st)
{
    const int64_t grid = (n + kFlashBlock - 1) / kFlashBlock;
    flashKernel<NC><<<unsigned(grid), kFlashBlock, 0, st>>>(ctx->fluid, n, P, T, z, sal, out, ctx->evalCounter);
    return 0;
}

template <int NC>
int launchEos(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *x,
              const int8_t *role, const double *sal, double *Z, double *lnphi, cudaStream_t st)
{
    const int64_t grid = (n + 255) / 256;
    eosKernel<NC><<<unsigned(grid), 256, 0, st>>>(ctx->fluid, n, P, T, x, role, sal, Z, lnphi);
    return 0;
}

template <int NC>
int launchStability(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                    const double *sal, const uint8_t *active, const double *comps, uint8_t *stable,
                    uint8_t *valid, uint8_t *mask, double *ts, double *inc, cudaStream_t st)
{
    const int64_t grid = (n + kFlashBlock - 1) / kFlashBlock;
    stabilityKernel<NC><<<unsigned(grid), kFlashBlock, 0, st>>>(ctx->fluid, n, P, T, z, sal, active, comps,
                                                               stable, valid, mask, ts, inc);
    return 0;
}

} // namespace nz
