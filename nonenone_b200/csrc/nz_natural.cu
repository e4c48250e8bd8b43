// nz_natural.cu -- Natural assembly entry points (state update, residual,
// Jacobian).  Until the device kernels land these refuse with
// NZ_ERR_UNSUPPORTED; there is no host fallback.
#include "common.cuh"

using namespace nz;

extern "C" {
int nz_natural_create(nz_ctx *, const nz_natural_desc *, nz_natural **out)
{
    if (out)
        *out = nullptr;
    return setError(NZ_ERR_UNSUPPORTED, "nz_natural_create: Natural assembly is not built yet");
}
int nz_natural_destroy(nz_natural *) { return NZ_OK; }
int nz_natural_pattern(nz_natural *, int64_t *, int64_t *, int64_t *)
{
    return setError(NZ_ERR_UNSUPPORTED, "Natural assembly is not built yet");
}
int nz_natural_set_history(nz_natural *, const double *, const double *, void *)
{
    return setError(NZ_ERR_UNSUPPORTED, "Natural assembly is not built yet");
}
int nz_update_state(nz_natural *, double *, double *, nz_report *, void *)
{
    return setError(NZ_ERR_UNSUPPORTED, "Natural assembly is not built yet");
}
int nz_residual(nz_natural *, const double *, const double *, double *, void *)
{
    return setError(NZ_ERR_UNSUPPORTED, "Natural assembly is not built yet");
}
int nz_jacobian(nz_natural *, const double *, const double *, double *, double *, void *)
{
    return setError(NZ_ERR_UNSUPPORTED, "Natural assembly is not built yet");
}
}
