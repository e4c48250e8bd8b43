// common.cuh -- shared host-side definitions of the CUDA library.
#pragma once

#include "../../include/nonenone_b200.h"
#include "eos.cuh"
#include "fluid_dev.cuh"

#include <cstdarg>
#include <cuda_runtime.h>

namespace nz
{

constexpr int kFlashBlock = 128;
// nz_ctx::evalCounter block: the EOS evaluation count (8 bytes), then the
// last batch's two self-check words (queue bound, spin guard).
constexpr size_t kCounterBlockBytes = 16;
constexpr int kTrialBlock = 128;
constexpr int kTrialBlocksPerSm = 8;

int setError(int code, const char *fmt, ...);
int cudaFail(cudaError_t e, const char *what);

inline bool ncSupported(int nc) { return nc == 3 || nc == 4 || nc == 5 || nc == 6 || nc == 8; }

} // namespace nz

// The opaque context behind nz_ctx*.
struct nz_ctx
{
    int device{0};
    nz_fluid_desc desc{};
    nz_flash_options options{};
    nz::FluidDev fluid{};
    unsigned long long *evalCounter{nullptr};   // EOS evaluations of the last flash batch
    int *checkWords{nullptr};                   // its self-check words (inside the evalCounter block)
    cudaStream_t ownStream{nullptr};
    int smCount{148};
    void *scratch{nullptr};                     // staged-flash work space (grow only)
    size_t scratchBytes{0};

    // Make the work space at least `bytes` large (cudaMalloc on growth only).
    int ensureScratch(size_t bytes);

    cudaStream_t hostStream()
    {
        if (!ownStream)
            cudaStreamCreateWithFlags(&ownStream, cudaStreamNonBlocking);
        return ownStream;
    }
};

namespace nz
{
template <int NC>
int launchStaged(nz_ctx *ctx, int64_t n, const double *P, const double *T, const double *z,
                 const double *sal, const nz_flash_out &out, bool mixed, cudaStream_t st);
// The staged flash into a caller-provided work space of `capacity` bytes.
template <int NC>
int launchStagedInto(nz_ctx *ctx, void *scratch, size_t capacity, int64_t n, const double *P, const double *T,
                     const double *z, const double *sal, const nz_flash_out &out, bool mixed, cudaStream_t st);
// Work-space bytes of an n-point staged flash, and the largest n that fits.
size_t stagedScratchBytesFor(int nc, int64_t n, const FluidDev &F);
int64_t stagedMaxPointsFor(int nc, size_t capacity, const FluidDev &F);
template <int NC>
size_t stagedScratchBytesNc(int64_t n, const FluidDev &F);
// The staged launch sequence (defined in staged_inst.cu) for callers in other
// translation units; the scratch block holds stagedScratchBytesNc<NC>(n) bytes.
template <int NC>
int stagedLaunchExt(const FluidDev &F, void *scratch, int64_t n, const double *P, const double *T,
                    const double *z, const double *sal, const nz_flash_out &out,
                    unsigned long long *evalCounter, int smCount, cudaStream_t st, bool mixed);
}

// Runtime nc -> compile-time NC dispatch over the instantiated component counts.
#define DISPATCH_NC(ncv, fn, ...)                                                  \
    do                                                                             \
    {                                                                              \
        int _rc = NZ_ERR_UNSUPPORTED;                                              \
        switch (ncv)                                                               \
        {                                                                          \
        case 3: _rc = fn<3>(__VA_ARGS__); break;                                   \
        case 4: _rc = fn<4>(__VA_ARGS__); break;                                   \
        case 5: _rc = fn<5>(__VA_ARGS__); break;                                   \
        case 6: _rc = fn<6>(__VA_ARGS__); break;                                   \
        case 8: _rc = fn<8>(__VA_ARGS__); break;                                   \
        default: return nz::setError(NZ_ERR_UNSUPPORTED, "nc=%d not compiled", int(ncv)); \
        }                                                                          \
        if (_rc != 0)                                                              \
            return _rc;                                                            \
    } while (0)
