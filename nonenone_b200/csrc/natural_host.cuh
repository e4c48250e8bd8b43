// natural_host.cuh -- host-side declarations of the Natural launchers.
#pragma once

#include "common.cuh"
#include "natural.cuh"

namespace nz
{
enum NatOp
{
    NAT_CACHE = 0,
    NAT_RESIDUAL = 1,
    NAT_JACOBIAN = 2,
    NAT_HISTORY = 3,
    NAT_UPDATE = 4,
    NAT_INIT = 5,
};

struct NatLaunch
{
    FluidDev F;
    NatConst K;
    NatGeom g;
    const double *primary;
    const double *ps;
    double *residual;
    double *values;
    double *prevAcc;
    double *newPrimary;
    double *newPs;
    uint8_t *status;
    unsigned long long *firstFailure;
    int *flag;
    const double *initP;   // NAT_INIT: P[ncell], z[ncell][nc]
    const double *initZ;
};

template <int NC>
int natLaunch(int op, const NatLaunch &a, cudaStream_t st);
} // namespace nz
