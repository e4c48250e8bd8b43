// natural_kernels.cuh -- per-cell Natural work and the kernels that run it.
//
// The per-cell functions are __host__-compilable like the flash headers, so a
// host build of exactly this code can be compared with the reference.
//
//   cell values      buildCellCache_ (natural_petsc_runtime_cell_cache.inc:66-116):
//                    properties of every cell, kept as the frozen exterior
//                    side of its faces (face_flux.hpp:54-63)
//   residual         formFunction (natural_petsc_runtime_residual.inc:59-120)
//   Jacobian         assembleJacobian_ / prepareFaceJacobianRowsAndAccumulateSelf_
//                    (natural_petsc_runtime_jacobian.inc:24-91,120-299): self
//                    block plus, per face, the reciprocal block (row = neighbour,
//                    column = this cell), mass rows only, negated
//   history          refreshPreviousPropertiesCache_
//                    (natural_petsc_runtime_cache_history.inc:180-262)
//   state update     updateStateWithReport (natural_petsc_runtime_state.inc:166-345)
#pragma once

#include "natural_state.cuh"

namespace nz
{

// Frozen-exterior cache fields: p, density[3], saturation[3], mobility[3], w[3][NC]
template <int NC>
struct CacheLayout
{
    static constexpr int p = 0;
    static constexpr int density = 1;
    static constexpr int saturation = 4;
    static constexpr int mobility = 7;
    static constexpr int w = 10;
    static constexpr int fields = 10 + 3 * NC;
};

template <int NC>
NZ_HDI void loadSide(const double *cache, int64_t ncell, int64_t c, FaceSide<NC> &s)
{
    using CL = CacheLayout<NC>;
    s.p = cache[CL::p * ncell + c];
    for (int ph = 0; ph < 3; ++ph)
    {
        s.density[ph] = cache[(CL::density + ph) * ncell + c];
        s.saturation[ph] = cache[(CL::saturation + ph) * ncell + c];
        s.mobility[ph] = cache[(CL::mobility + ph) * ncell + c];
        for (int i = 0; i < NC; ++i)
            s.w[ph][i] = cache[(CL::w + ph * NC + i) * ncell + c];
    }
}

// Properties of cell c, values only (false where the reference throws).
template <int NC>
NZ_HD bool cellValues(const FluidDev &F, const NatConst &K, const NatGeom &g, const double *primary, const double *ps,
                      int64_t c, CellStateT<NC, Val> &st, CellPropsT<NC, Val> &pr)
{
    using L = Layout<NC>;
    decodeCell<NC, Val>(primary + c * L::B, ps[c * L::NPS + L::psFlag], -1, st);
    if (st.presence == 0)   // decodePhasePresence throws (phase_behavior.hpp:81-87)
        return false;
    return cellProperties<NC, Val>(F, K, st, g.porosity[c], pr);
}

template <int NC>
NZ_HD void toSide(const CellStateT<NC, Val> &st, const CellPropsT<NC, Val> &pr, FaceSide<NC> &s)
{
    s.p = st.p.v;
    for (int ph = 0; ph < 3; ++ph)
    {
        s.density[ph] = pr.density[ph].v;
        s.saturation[ph] = pr.saturation[ph].v;
        s.mobility[ph] = pr.mobility[ph].v;
        for (int i = 0; i < NC; ++i)
            s.w[ph][i] = pr.w[ph][i].v;
    }
}

template <int NC>
NZ_HD bool cellCacheStore(const FluidDev &F, const NatConst &K, const NatGeom &g, const double *primary,
                          const double *ps, int64_t c)
{
    using CL = CacheLayout<NC>;
    CellStateT<NC, Val> st;
    CellPropsT<NC, Val> pr;
    const bool ok = cellValues<NC>(F, K, g, primary, ps, c, st, pr);
    FaceSide<NC> s;
    toSide<NC>(st, pr, s);
    const int64_t n = g.ncell;
    g.cache[CL::p * n + c] = s.p;
    for (int ph = 0; ph < 3; ++ph)
    {
        g.cache[(CL::density + ph) * n + c] = s.density[ph];
        g.cache[(CL::saturation + ph) * n + c] = s.saturation[ph];
        g.cache[(CL::mobility + ph) * n + c] = s.mobility[ph];
        for (int i = 0; i < NC; ++i)
            g.cache[(CL::w + ph * NC + i) * n + c] = s.w[ph][i];
    }
    return ok;
}

// Residual block of cell c: local equations plus the summed outward face fluxes.
template <int NC>
NZ_HD bool cellResidual(const FluidDev &F, const NatConst &K, const NatGeom &g, const double *primary,
                        const double *ps, int64_t c, double *out)
{
    using L = Layout<NC>;
    CellStateT<NC, Val> st;
    CellPropsT<NC, Val> pr;
    if (!cellValues<NC>(F, K, g, primary, ps, c, st, pr))
        return false;
    Val res[L::B];
    localResidual<NC, Val>(K, st, pr, g.prevAcc + c * NC, g.volume[c], res);
    FaceSide<NC> in;
    toSide<NC>(st, pr, in);
    double outward[NC];
    for (int i = 0; i < NC; ++i)
        outward[i] = 0.0;
    for (int64_t j = g.offset[c]; j < g.offset[c + 1]; ++j)
    {
        const int64_t nb = g.neighbor[j];
        FaceSide<NC> ex;
        loadSide<NC>(g.cache, g.ncell, nb, ex);
        double flux[NC];
        faceFluxValue<NC>(in, ex, g.trans[j], g.gravity[j], g.volume[c], g.volume[nb], c, nb, flux);
        for (int i = 0; i < NC; ++i)
            outward[i] += flux[i];
    }
    for (int i = 0; i < NC; ++i)
        res[L::mass + i] += outward[i];
    for (int r = 0; r < L::B; ++r)
        out[c * L::B + r] = res[r].v;
    return true;
}

// Column k of cell c's Jacobian blocks (direction k seeded).  Writes column k
// of the self block and of every reciprocal block of c's faces; with
// `residual` set, the lane of direction 0 also writes the residual block.
template <int NC>
NZ_HD bool cellJacobianColumn(const FluidDev &F, const NatConst &K, const NatGeom &g, const double *primary,
                              const double *ps, int64_t c, int k, double *values, double *residual)
{
    using L = Layout<NC>;
    constexpr int B = L::B;
    CellStateT<NC, Dual> st;
    decodeCell<NC, Dual>(primary + c * B, ps[c * L::NPS + L::psFlag], k, st);
    CellPropsT<NC, Dual> pr;
    if (st.presence == 0 || !cellProperties<NC, Dual>(F, K, st, g.porosity[c], pr))
        return false;
    Dual res[B];
    localResidual<NC, Dual>(K, st, pr, g.prevAcc + c * NC, g.volume[c], res);
    // Derivatives: each face's row is added into the self block in face order
    // (jacobian.inc:120-237).  Values (lane 0, when asked): the residual's
    // value flux, summed and then added to the local block (residual.inc:59-120).
    const bool wantResidual = residual && k == 0;
    FaceSide<NC> inVal;
    if (wantResidual)
    {
        inVal.p = st.p.v;
        for (int ph = 0; ph < 3; ++ph)
        {
            inVal.density[ph] = pr.density[ph].v;
            inVal.saturation[ph] = pr.saturation[ph].v;
            inVal.mobility[ph] = pr.mobility[ph].v;
            for (int i = 0; i < NC; ++i)
                inVal.w[ph][i] = pr.w[ph][i].v;
        }
    }
    double outward[NC];
    for (int i = 0; i < NC; ++i)
        outward[i] = 0.0;
    for (int64_t j = g.offset[c]; j < g.offset[c + 1]; ++j)
    {
        const int64_t nb = g.neighbor[j];
        FaceSide<NC> ex;
        loadSide<NC>(g.cache, g.ncell, nb, ex);
        Dual flux[NC];
        faceFlux<NC, Dual>(st, pr, ex, g.trans[j], g.gravity[j], g.volume[c], g.volume[nb], c, nb, flux);
        double *recip = values + connBlock(g, c, j) * (B * B);
        for (int r = 0; r < B; ++r)
            recip[r * B + k] = r < NC ? -flux[r].d : 0.0;
        for (int i = 0; i < NC; ++i)
            res[L::mass + i].d += flux[i].d;
        if (wantResidual)
        {
            double fv[NC];
            faceFluxValue<NC>(inVal, ex, g.trans[j], g.gravity[j], g.volume[c], g.volume[nb], c, nb, fv);
            for (int i = 0; i < NC; ++i)
                outward[i] += fv[i];
        }
    }
    double *self = values + selfBlock(g, c) * (B * B);
    for (int r = 0; r < B; ++r)
        self[r * B + k] = res[r].d;
    if (wantResidual)
    {
        for (int i = 0; i < NC; ++i)
            res[L::mass + i].v += outward[i];
        for (int r = 0; r < B; ++r)
            residual[c * B + r] = res[r].v;
    }
    return true;
}

// History: accumulation of the accepted state.
template <int NC>
NZ_HD bool cellHistory(const FluidDev &F, const NatConst &K, const NatGeom &g, const double *primary,
                       const double *ps, int64_t c, double *prevAcc)
{
    CellStateT<NC, Val> st;
    CellPropsT<NC, Val> pr;
    const bool ok = cellValues<NC>(F, K, g, primary, ps, c, st, pr);
    for (int i = 0; i < NC; ++i)
        prevAcc[c * NC + i] = ok ? accumulation<NC, Val>(pr, i).v : 0.0;
    return ok;
}

// Status byte of one cell's phase-state update: bits 0-1 the PhaseUpdateStatus,
// bits 2-6 the five report flags.
NZ_BOTH uint8_t packOutcome(const UpdateOutcome &o)
{
    return uint8_t(o.status | (o.phaseRemoved << 2) | (o.missingPhaseUnstable << 3) | (o.stabilityInvalid << 4) |
                   (o.restrictedFailed << 5) | (o.unrestrictedFailed << 6));
}

// sanitizePrimaryBeforeFlash + updatePhaseState of cell c into the scratch copy.
// With width > 1, `width` lanes run the cell in lockstep and split the seeds of
// its stability tests; lane 0 writes.  With `memo` / `flashMemo`, a stability
// test or top-level flash whose input matches memo[c] / flashMemo[c] takes its
// stored answer.
template <int NC>
NZ_HD uint8_t cellUpdate(const FluidDev &F, const NatConst &K, const double *primary, const double *ps, int64_t c,
                         double *newPrimary, double *newPs, int lane = 0, int width = 1,
                         StabilityMemo<NC> *memo = nullptr, const FlashMemo<NC> *flashMemo = nullptr)
{
    using L = Layout<NC>;
    double a[L::B];
    for (int r = 0; r < L::B; ++r)
        a[r] = primary[c * L::B + r];
    PhaseRec<NC> rec;
    if (!decodePhaseRec<NC>(ps + c * L::NPS, rec))   // invalid presence flag: the reference throws
        return packOutcome(UpdateOutcome{UPD_FAILED, false, false, false, false, false});
    Equilibrium<NC> eq;
    eq.s.setup(&F, F.salinity);
    eq.s.lane = lane;
    eq.s.width = width;
    eq.s.stabMemo = memo ? memo + c : nullptr;
    eq.s.flashMemo = flashMemo ? flashMemo + c : nullptr;
    eq.K = &K;
    eq.sanitize(a);
    UpdateOutcome o = eq.update(a, rec);
    if (eq.s.err)
        o = UpdateOutcome{UPD_FAILED, false, false, false, false, false};
    if (o.status != UPD_FAILED && lane == 0)
    {
        for (int r = 0; r < L::B; ++r)
            newPrimary[c * L::B + r] = a[r];
        encodePhaseRec<NC>(rec, newPs + c * L::NPS);
    }
    return packOutcome(o);
}

// The head of cell c's update (decode, sanitize, updateHead) without any
// flash or stability test: the input of the main-path stability test.  False
// when the phase state cannot be decoded or a composition not normalised.
template <int NC>
NZ_HD bool cellUpdateHead(const FluidDev &F, const NatConst &K, const double *primary, const double *ps, int64_t c,
                          UpdateHead<NC> &h)
{
    using L = Layout<NC>;
    double a[L::B];
    for (int r = 0; r < L::B; ++r)
        a[r] = primary[c * L::B + r];
    PhaseRec<NC> rec;
    if (!decodePhaseRec<NC>(ps + c * L::NPS, rec))
        return false;
    Equilibrium<NC> eq;
    eq.s.setup(&F, F.salinity);
    eq.K = &K;
    eq.sanitize(a);
    return eq.updateHead(a, rec, h);
}

// initializeUniformFromPTZ per cell (natural_petsc_runtime_state.inc:107-164):
// flashPTZ, then assignFlashResult into a default phase state.  False where the
// flash does not converge (the reference throws).
template <int NC>
NZ_HD bool cellInitPtz(const FluidDev &F, const NatConst &K, const double *P, const double *z, int64_t c,
                       double *primary, double *ps, int lane = 0, int width = 1,
                       const FlashMemo<NC> *memo = nullptr)
{
    using L = Layout<NC>;
    Equilibrium<NC> eq;
    eq.s.setup(&F, F.salinity);
    eq.s.lane = lane;
    eq.s.width = width;
    eq.s.flashMemo = memo;   // the batched flash's answer for this cell's input, if given
    eq.K = &K;
    Result<NC> r;
    eq.s.template flash<true>(P[c], K.temperature, z + c * NC, r);
    if (!r.converged || eq.s.err)
        return false;
    double a[L::B];
    for (int k = 0; k < L::B; ++k)
        a[k] = 0.0;
    a[0] = P[c];
    PhaseRec<NC> rec;   // PhaseStateData defaults (phase_state_data.hpp)
    rec.presence = ALL_BITS;
    rec.suppression = 0;
    for (int i = 0; i < NC; ++i)
        rec.Kg[i] = rec.Kw[i] = rec.z[i] = 0.0;
    rec.beta[0] = 1.0;
    rec.beta[1] = rec.beta[2] = 0.0;
    rec.Z[0] = rec.Z[1] = rec.Z[2] = 1.0;
    eq.assignFlashResult(a, rec, r);
    if (eq.s.err)
        return false;
    if (lane != 0)
        return true;
    for (int k = 0; k < L::B; ++k)
        primary[c * L::B + k] = a[k];
    encodePhaseRec<NC>(rec, ps + c * L::NPS);
    return true;
}

#ifdef __CUDACC__
// ------------------------------------------------------------------ kernels --
constexpr int kNatBlock = 128;

template <int NC>
__global__ void __launch_bounds__(kNatBlock) natCacheKernel(const __grid_constant__ FluidDev F,
                                                            const __grid_constant__ NatConst K, NatGeom g,
                                                            const double *primary, const double *ps, int *flag)
{
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= g.ncell)
        return;
    if (!cellCacheStore<NC>(F, K, g, primary, ps, c))
        atomicOr(flag, 1);
}

template <int NC>
__global__ void __launch_bounds__(kNatBlock) natResidualKernel(const __grid_constant__ FluidDev F,
                                                               const __grid_constant__ NatConst K, NatGeom g,
                                                               const double *primary, const double *ps,
                                                               double *residual, int *flag)
{
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= g.ncell)
        return;
    if (!cellResidual<NC>(F, K, g, primary, ps, c, residual))
        atomicOr(flag, 1);
}

// B lanes per cell, floor(32 / B) cells per warp.
template <int NC>
__global__ void __launch_bounds__(kNatBlock) natJacobianKernel(const __grid_constant__ FluidDev F,
                                                               const __grid_constant__ NatConst K, NatGeom g,
                                                               const double *primary, const double *ps,
                                                               double *values, double *residual, int *flag)
{
    constexpr int B = Layout<NC>::B;
    constexpr int perWarp = 32 / B;
    const int lane = threadIdx.x & 31;
    const int warp = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int group = lane / B;
    const int k = lane - group * B;
    const int64_t c = int64_t(warp) * perWarp + group;
    if (group >= perWarp || c >= g.ncell)
        return;
    if (!cellJacobianColumn<NC>(F, K, g, primary, ps, c, k, values, residual))
        atomicOr(flag, 1);
}

// Lane layout of natJacobianKernelN with KD directions per lane.
template <int NC, int KD>
struct JacobianShape
{
    static constexpr int B = Layout<NC>::B;
    static constexpr int K = KD;                     // directions per lane
    static constexpr int G = (B + K - 1) / K;        // lanes per cell
    static constexpr int perWarp = 32 / G;           // cells per warp
    static constexpr int warps = kNatBlock / 32;
    static constexpr size_t smemBytes = size_t(warps) * perWarp * B * B * sizeof(double);
};

// The BAIJ Jacobian with K directions per lane (DualN<K>): G = ceil(B / K)
// lanes per cell, so the value part of a cell's properties -- transcendental
// heavy, and recomputed by every lane -- runs G times per cell instead of B.
// Every block of the warp's cells is assembled in shared memory and stored to
// its BAIJ slot as one contiguous B*B*8-byte range by the whole warp (whole
// 32-byte sectors), the reciprocal blocks face by face in connection order and
// the self block last, with the face rows added into it in the same order as
// the one-direction kernel (jacobian.inc:120-237).
template <int NC, int KDIR>
__global__ void __launch_bounds__(kNatBlock) natJacobianKernelN(const __grid_constant__ FluidDev F,
                                                                const __grid_constant__ NatConst K, NatGeom g,
                                                                const double *primary, const double *ps,
                                                                double *values, double *residual, int *flag)
{
    using L = Layout<NC>;
    using J = JacobianShape<NC, KDIR>;
    constexpr int B = L::B;
    constexpr int KD = J::K;
    constexpr int G = J::G;
    constexpr int perWarp = J::perWarp;
    constexpr int BB = B * B;
    using S = DualN<KD>;
    extern __shared__ double natTile[];
    const int lane = threadIdx.x & 31;
    const int warpInBlock = threadIdx.x >> 5;
    double *tile = natTile + size_t(warpInBlock) * perWarp * BB;
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int group = lane / G;
    const int sub = lane - group * G;
    const int k0 = sub * KD;
    const int64_t c = warp * perWarp + group;
    const bool mine = group < perWarp && c < g.ncell;

    CellStateT<NC, S> st;
    CellPropsT<NC, S> pr;
    S res[B];
    bool ok = false;
    if (mine)
    {
        decodeCell<NC, S>(primary + c * B, ps[c * L::NPS + L::psFlag], k0, st);
        ok = st.presence != 0 && cellProperties<NC, S>(F, K, st, g.porosity[c], pr);
        if (ok)
            localResidual<NC, S>(K, st, pr, g.prevAcc + c * NC, g.volume[c], res);
        else if (sub == 0)
            atomicOr(flag, 1);
    }
    const bool wantResidual = ok && residual && sub == 0;
    FaceSide<NC> inVal;
    if (wantResidual)
    {
        inVal.p = st.p.v;
        for (int ph = 0; ph < 3; ++ph)
        {
            inVal.density[ph] = pr.density[ph].v;
            inVal.saturation[ph] = pr.saturation[ph].v;
            inVal.mobility[ph] = pr.mobility[ph].v;
            for (int i = 0; i < NC; ++i)
                inVal.w[ph][i] = pr.w[ph][i].v;
        }
    }
    double outward[NC];
    for (int i = 0; i < NC; ++i)
        outward[i] = 0.0;
    const int64_t first = ok ? g.offset[c] : 0;
    const int nfaces = ok ? int(g.offset[c + 1] - first) : 0;
    int maxFaces = nfaces;
    for (int off = 16; off > 0; off >>= 1)
        maxFaces = max(maxFaces, __shfl_xor_sync(0xffffffffu, maxFaces, off));
    double *myTile = tile + (group < perWarp ? group : 0) * BB;

    // store the tiles of the warp's cells that have a block in this pass; the
    // loop runs the same number of times on every lane (the tiles' total need
    // not be a multiple of 32), so every shuffle has the whole warp
    auto flush = [&](bool has, int64_t slot) {
        __syncwarp();
        constexpr int total = perWarp * BB;
        for (int base = 0; base < total; base += 32)
        {
            const int e = base + lane;
            const int q = e < total ? e / BB : 0;
            const int o = e - q * BB;
            const int owner = q * G;
            const int qHas = __shfl_sync(0xffffffffu, int(has), owner);
            const long long qSlot = __shfl_sync(0xffffffffu, (long long)slot, owner);
            if (e < total && qHas)
                values[qSlot * BB + o] = tile[e];
        }
        __syncwarp();
    };

    for (int f = 0; f < maxFaces; ++f)
    {
        const bool has = f < nfaces;
        int64_t slot = 0;
        if (has)
        {
            const int64_t j = first + f;
            const int64_t nb = g.neighbor[j];
            FaceSide<NC> ex;
            loadSide<NC>(g.cache, g.ncell, nb, ex);
            S flux[NC];
            faceFlux<NC, S>(st, pr, ex, g.trans[j], g.gravity[j], g.volume[c], g.volume[nb], c, nb, flux);
            for (int i = 0; i < NC; ++i)
                for (int jj = 0; jj < KD; ++jj)
                    res[L::mass + i].d[jj] += flux[i].d[jj];
            for (int r = 0; r < B; ++r)
                for (int jj = 0; jj < KD; ++jj)
                    if (k0 + jj < B)
                        myTile[r * B + k0 + jj] = r < NC ? -flux[r].d[jj] : 0.0;
            slot = connBlock(g, c, j);
            if (wantResidual)
            {
                double fv[NC];
                faceFluxValue<NC>(inVal, ex, g.trans[j], g.gravity[j], g.volume[c], g.volume[nb], c, nb, fv);
                for (int i = 0; i < NC; ++i)
                    outward[i] += fv[i];
            }
        }
        flush(has, slot);
    }
    if (ok)
        for (int r = 0; r < B; ++r)
            for (int jj = 0; jj < KD; ++jj)
                if (k0 + jj < B)
                    myTile[r * B + k0 + jj] = res[r].d[jj];
    flush(ok, ok ? selfBlock(g, c) : 0);
    if (wantResidual)
    {
        for (int i = 0; i < NC; ++i)
            res[L::mass + i].v += outward[i];
        for (int r = 0; r < B; ++r)
            residual[c * B + r] = res[r].v;
    }
}

template <int NC>
__global__ void __launch_bounds__(kNatBlock) natHistoryKernel(const __grid_constant__ FluidDev F,
                                                              const __grid_constant__ NatConst K, NatGeom g,
                                                              const double *primary, const double *ps,
                                                              double *prevAcc, int *flag)
{
    const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (c >= g.ncell)
        return;
    if (!cellHistory<NC>(F, K, g, primary, ps, c, prevAcc))
        atomicOr(flag, 1);
}

// Width 32: one warp per cell, the lanes splitting the seeds of the cell's
// stability tests (short latency, for grids too small to fill the GPU).
// Width 1: one thread per cell (a warp's lanes hold 32 cells, so the solver's
// per-lane stack is shared by 32 times fewer cells in flight).
template <int NC>
__global__ void __launch_bounds__(kNatBlock) natUpdateKernel(const __grid_constant__ FluidDev F,
                                                             const __grid_constant__ NatConst K, int64_t ncell,
                                                             const double *primary, const double *ps,
                                                             double *newPrimary, double *newPs, uint8_t *status,
                                                             unsigned long long *firstFailure, int width,
                                                             StabilityMemo<NC> *memo, const FlashMemo<NC> *flashMemo)
{
    const int lane = width == 32 ? int(threadIdx.x & 31) : 0;
    const int64_t c = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / width;
    if (c >= ncell)
        return;
    const uint8_t s = cellUpdate<NC>(F, K, primary, ps, c, newPrimary, newPs, lane, width, memo, flashMemo);
    if (lane != 0)
        return;
    status[c] = s;
    if ((s & 3) == UPD_FAILED)
        atomicMin(firstFailure, (unsigned long long)c);
}

// Width 32 or 1, as the update.
template <int NC>
__global__ void __launch_bounds__(kNatBlock) natInitKernel(const __grid_constant__ FluidDev F,
                                                           const __grid_constant__ NatConst K, int64_t ncell,
                                                           const double *P, const double *z, double *primary,
                                                           double *ps, unsigned long long *firstFailure, int width,
                                                           const FlashMemo<NC> *memos)
{
    const int lane = width == 32 ? int(threadIdx.x & 31) : 0;
    const int64_t c = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) / width;
    if (c >= ncell)
        return;
    if (!cellInitPtz<NC>(F, K, P, z, c, primary, ps, lane, width, memos ? memos + c : nullptr) && lane == 0)
        atomicMin(firstFailure, (unsigned long long)c);
}
#endif


} // namespace nz
