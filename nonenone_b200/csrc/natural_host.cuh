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
    NAT_UPDATE_PREPARE = 6,   // staged update: main-path stability tests, list of reflash cells
    NAT_UPDATE_REFLASH = 7,   // staged update: batched flash of the listed cells
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
    void *stagedScratch;   // staged update: natStagedBytesNc<NC> bytes, or null for the per-cell update
    void *flashScratch;    // NAT_UPDATE_REFLASH: natReflashBytesNc<NC>(reflashCount) bytes;
                           // NAT_INIT: natInitBytesNc<NC>(ncell) bytes, or null for the per-cell flash
    int reflashCount;
};

template <int NC>
int natLaunch(int op, const NatLaunch &a, cudaStream_t st);

// Work space of the staged phase-state update of n cells, and of its batched
// reflash of n cells; device address of the reflash count inside the former.
template <int NC>
size_t natStagedBytesNc(int64_t n, const FluidDev &F);
template <int NC>
size_t natReflashBytesNc(int64_t n, const FluidDev &F);
template <int NC>
int *natReflashCountNc(void *scratch, int64_t n, const FluidDev &F);
// Work space of the batched P-T-z initialisation of n cells.
template <int NC>
size_t natInitBytesNc(int64_t n, const FluidDev &F);
} // namespace nz
