// flash_inst.cu -- the one-thread-per-point flash, EOS and stability kernels of
// one component count.  Every *_inst.cu unit is compiled once per NZ_INST_NC
// value (3, 4, 5, 6, 8), so the heavy device code of each component count and
// kernel family builds in its own translation unit.
#include "flash_kernels.cuh"

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
} // namespace nz
