// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A PETSc-free harness around the reference's own FP64 C++ code
// (MPMC_SCW models/include/natural/...).  It is compiled against the
// reference headers where they lie (see oracle/Makefile) into
// oracle/_ref/libnzref.so and is used by tests/ as the parity checker and by
// bench.py as the timed CPU baseline.  Nothing in the product links it.
//
// What is restated here is only the loop structure of the reference runtime:
//   * flash batch            -> CubicThreePhaseFlash::flash per point
//                               (models/include/natural/thermo/three_phase_flash.hpp:83-227)
//   * updateStateWithReport  -> natural_petsc_runtime_state.inc:166-345
//   * formFunction           -> natural_petsc_runtime_residual.inc:19-133
//                               + natural_petsc_runtime_cell_cache.inc:8-185
//   * assembleJacobian_      -> natural_petsc_runtime_jacobian.inc:8-299
//   * previous accumulation  -> natural_petsc_runtime_cache_history.inc:180-262
//   * boundary distance      -> the trial loop of stabilityTest
//                               (three_phase_flash.hpp:399-480), non-trivial trials only
// Every physical computation is a call into the reference's own headers.
#include <indices/indices.hpp>
#include <natural/fluid_system.hpp>
#include <natural/kernel/cell_kernel.hpp>
#include <natural/state/three_phase_equilibrium.hpp>
#include <natural/thermo/three_phase_flash.hpp>
#include <natural/petsc/phase_state_codec.hpp>
#include <natural/petsc/property_conversion.hpp>

#include "../include/nonenone_b200.h"

#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace
{
using namespace MPMC;

thread_local std::string g_error;

template <int NC>
using Config = CompositionalModelConfig<
    NC, true, false, false, false, false,
    PhaseBehaviorModel::FullyCompositionalThreePhase>;
template <int NC>
using SIdx = ScalarIndices<Config<NC>>;
template <int NC>
using AIdx = ADIndices<Config<NC>>;

double swBip(const nz_fluid_desc &d, int component, double temperature, double salinity)
{
    switch (d.sw_bip_kind[component])
    {
    case NZ_SW_BIP_CONSTANT:
        return d.sw_bip_value[component];
    case NZ_SW_BIP_CO2:
        return SoreideWhitsonCorrelations::co2AqueousBip(
            temperature, d.tc[component], salinity);
    case NZ_SW_BIP_HYDROCARBON:
        return SoreideWhitsonCorrelations::hydrocarbonAqueousBip(
            temperature, d.tc[component], d.acentric[component], salinity);
    case NZ_SW_BIP_CO2_CHABAB:
        return SoreideWhitsonCorrelations::co2AqueousBipChabab2019(
            temperature, salinity);
    default:
        return d.kij[d.water_component * NZ_MAX_NC + component];
    }
}

// Builds the EOS the way case/include/case/fluid_factory.hpp:229-300 does.
template <class Indices>
CubicEquationOfState<Indices> makeEos(const nz_fluid_desc &d, double salinity)
{
    constexpr int N = Indices::numComponents;
    std::array<double, N> tc{}, pc{}, vc{}, om{}, mw{};
    std::array<std::array<double, N>, N> k{};
    for (int i = 0; i < N; ++i)
    {
        tc[i] = d.tc[i];
        pc[i] = d.pc[i];
        vc[i] = d.vc[i];
        om[i] = d.acentric[i];
        mw[i] = d.mw[i];
        for (int j = 0; j < N; ++j)
            k[i][j] = d.kij[i * NZ_MAX_NC + j];
    }
    CompositionalMixture<Indices> mixture(tc, pc, vc, om, mw, k);
    CubicEquationOfState<Indices> eos(
        d.omega_a, d.omega_b, std::move(mixture), d.eos_type, d.m1, d.m2,
        d.minimum_composition);
    if (d.eos_model == NZ_EOS_SW)
    {
        typename CubicEquationOfState<Indices>::SoreideWhitsonOptions sw;
        sw.waterComponent = d.water_component;
        sw.salinityMolality = salinity;
        for (int c = 0; c < N; ++c)
        {
            if (d.sw_bip_kind[c] == NZ_SW_BIP_KIJ)
                continue;
            const nz_fluid_desc copy = d;
            sw.aqueousWaterBip[static_cast<std::size_t>(c)] =
                [copy, c](double temperature, double s) {
                    return swBip(copy, c, temperature, s);
                };
        }
        eos.configureSoreideWhitson(std::move(sw));
    }
    else if (d.eos_model == NZ_EOS_CPA)
    {
        // CubicPlusAssociationOptions filled as case/include/case/fluid_factory.hpp:323-396 does
        typename CubicEquationOfState<Indices>::CubicPlusAssociationOptions cpa;
        for (int c = 0; c < N; ++c)
        {
            const auto cc = static_cast<std::size_t>(c);
            cpa.a0[cc] = d.cpa_a0[c];
            cpa.b[cc] = d.cpa_b[c];
            cpa.c1[cc] = d.cpa_c1[c];
            cpa.associationEnergy[cc] = d.cpa_epsilon[c];
            cpa.associationVolume[cc] = d.cpa_beta[c];
            cpa.donorSites[cc] = d.cpa_donor_sites[c];
            cpa.acceptorSites[cc] = d.cpa_acceptor_sites[c];
            for (int j = 0; j < N; ++j)
            {
                cpa.crossAssociationEnergy[cc][static_cast<std::size_t>(j)] = d.cpa_cross_epsilon[c * NZ_MAX_NC + j];
                cpa.crossAssociationVolume[cc][static_cast<std::size_t>(j)] = d.cpa_cross_beta[c * NZ_MAX_NC + j];
            }
        }
        cpa.physicalTerm = d.cpa_physical_term == NZ_CPA_PR ? CpaCubicPhysicalTerm::PengRobinson
                                                            : CpaCubicPhysicalTerm::SoaveRedlichKwong;
        cpa.radialDistribution = d.cpa_radial == NZ_CPA_RADIAL_CARNAHAN_STARLING
            ? CpaRadialDistribution::CarnahanStarling
            : CpaRadialDistribution::Simplified;
        cpa.maximumAssociationIterations = d.cpa_max_association_iterations;
        cpa.associationTolerance = d.cpa_association_tolerance;
        cpa.associationDamping = d.cpa_association_damping;
        eos.configureCubicPlusAssociation(std::move(cpa));
    }
    else if (d.eos_model != NZ_EOS_PR)
    {
        throw std::invalid_argument("oracle: unknown eos_model");
    }
    return eos;
}

ThreePhaseFlashOptions toOptions(const nz_flash_options *o, int water)
{
    ThreePhaseFlashOptions r;
    r.waterComponent = water;
    if (o == nullptr)
        return r;
    r.maximumIterations = o->maximum_iterations;
    r.maximumRachfordRiceIterations = o->maximum_rachford_rice_iterations;
    r.maximumStabilityIterations = o->maximum_stability_iterations;
    r.stabilitySsiIterationsBeforeNewton = o->stability_ssi_before_newton;
    r.maximumStabilityNewtonIterations = o->maximum_stability_newton;
    r.twoPhaseSsiIterationsBeforeNewton = o->two_phase_ssi_before_newton;
    r.maximumTwoPhaseNewtonIterations = o->maximum_two_phase_newton;
    r.threePhaseSsiIterationsBeforeNewton = o->three_phase_ssi_before_newton;
    r.maximumThreePhaseNewtonIterations = o->maximum_three_phase_newton;
    r.fugacityTolerance = o->fugacity_tolerance;
    r.rachfordRiceTolerance = o->rachford_rice_tolerance;
    r.stabilityTolerance = o->stability_tolerance;
    r.phaseFractionTolerance = o->phase_fraction_tolerance;
    r.coincidentPhaseCompositionTolerance = o->coincident_composition_tolerance;
    r.compositionFloor = o->composition_floor;
    r.logKStepLimit = o->log_k_step_limit;
    r.numericalJacobianStep = o->numerical_jacobian_step;
    return r;
}

template <class F>
void parallelFor(int64_t n, int threads, F &&body)
{
    if (threads <= 1 || n < 2)
    {
        body(int64_t(0), n, 0);
        return;
    }
    threads = static_cast<int>(std::min<int64_t>(threads, n));
    std::vector<std::thread> pool;
    const int64_t chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t)
    {
        const int64_t b = t * chunk;
        const int64_t e = std::min(n, b + chunk);
        if (b >= e)
            break;
        pool.emplace_back([&, b, e, t]() { body(b, e, t); });
    }
    for (auto &th : pool)
        th.join();
}

// ---------------------------------------------------------------- flash ----
template <int NC>
int flashBatch(const nz_fluid_desc *d, const nz_flash_options *o, int64_t n,
               const double *P, const double *T, const double *z,
               const double *salinity, const nz_flash_out *out, int threads)
{
    using I = SIdx<NC>;
    using Flash = CubicThreePhaseFlash<I>;
    const auto options = toOptions(o, d->water_component);
    const bool perPointEos = d->eos_model == NZ_EOS_SW && salinity != nullptr;
    std::atomic<int> fatal{0};

    parallelFor(n, threads, [&](int64_t b, int64_t e, int) {
        std::unique_ptr<CubicEquationOfState<I>> shared;
        std::unique_ptr<Flash> sharedFlash;
        if (!perPointEos)
        {
            shared = std::make_unique<CubicEquationOfState<I>>(makeEos<I>(*d, d->sw_salinity));
            sharedFlash = std::make_unique<Flash>(*shared, options);
        }
        for (int64_t i = b; i < e; ++i)
        {
            std::unique_ptr<CubicEquationOfState<I>> local;
            std::unique_ptr<Flash> localFlash;
            Flash *flash = sharedFlash.get();
            if (perPointEos)
            {
                local = std::make_unique<CubicEquationOfState<I>>(makeEos<I>(*d, salinity[i]));
                localFlash = std::make_unique<Flash>(*local, options);
                flash = localFlash.get();
            }
            std::array<double, NC> zi{};
            for (int c = 0; c < NC; ++c)
                zi[c] = z[c * n + i];
            uint8_t status = NZ_FLASH_CONVERGED;
            typename Flash::Result r;
            try
            {
                r = flash->flash(P[i], T[i], zi);
                if (!r.converged)
                    status = NZ_FLASH_FAILED;
            }
            catch (const std::invalid_argument &)
            {
                status = NZ_FLASH_BAD_INPUT;
                r = typename Flash::Result{};
            }
            catch (const std::exception &)
            {
                status = NZ_FLASH_EOS_ERROR;
                r = typename Flash::Result{};
            }
            if (out->status) out->status[i] = status;
            if (out->presence) out->presence[i] = r.converged ? r.presence.bits() : 0;
            if (out->iterations) out->iterations[i] = r.iterations;
            for (int p = 0; p < 3; ++p)
            {
                if (out->beta) out->beta[p * n + i] = r.phaseMoleFraction[p];
                if (out->saturation) out->saturation[p * n + i] = r.saturation[p];
                if (out->compressibility) out->compressibility[p * n + i] = r.compressibility[p];
                if (out->molar_density) out->molar_density[p * n + i] = r.molarDensity[p];
                if (out->composition)
                    for (int c = 0; c < NC; ++c)
                        out->composition[(p * NC + c) * n + i] = r.composition[p][c];
            }
            for (int c = 0; c < NC; ++c)
            {
                if (out->k_gas_oil) out->k_gas_oil[c * n + i] = r.vaporOilK[c];
                if (out->k_water_oil) out->k_water_oil[c * n + i] = r.waterOilK[c];
            }
        }
    });
    return fatal.load();
}

template <int NC>
int eosBatch(const nz_fluid_desc *d, int64_t n, const double *P, const double *T,
             const double *x, const int8_t *role, const double *salinity,
             double *Z, double *lnphi)
{
    using I = SIdx<NC>;
    for (int64_t i = 0; i < n; ++i)
    {
        const auto eos = makeEos<I>(*d, salinity ? salinity[i] : d->sw_salinity);
        std::array<double, NC> xi{};
        for (int c = 0; c < NC; ++c)
            xi[c] = x[c * n + i];
        const auto phase = static_cast<CompositionalPhase>(role[i]);
        try
        {
            const auto r = eos.phaseResult(P[i], T[i], xi, phase);
            Z[i] = r.compressibility;
            for (int c = 0; c < NC; ++c)
                lnphi[c * n + i] = std::log(r.fugacityCoefficient[c]);
        }
        catch (const std::exception &)
        {
            Z[i] = std::nan("");
            for (int c = 0; c < NC; ++c)
                lnphi[c * n + i] = std::nan("");
        }
    }
    return 0;
}

template <int NC>
int stabilityBatch(const nz_fluid_desc *d, const nz_flash_options *o, int64_t n,
                   const double *P, const double *T, const double *z,
                   const double *salinity, const uint8_t *active,
                   const double *comps, uint8_t *stable, uint8_t *valid,
                   uint8_t *unstableMask, double *trialSum, double *incipient,
                   int threads)
{
    using I = SIdx<NC>;
    using Flash = CubicThreePhaseFlash<I>;
    const auto options = toOptions(o, d->water_component);
    parallelFor(n, threads, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i)
        {
            const auto eos = makeEos<I>(*d, salinity ? salinity[i] : d->sw_salinity);
            Flash flash(eos, options);
            std::array<double, NC> zi{};
            std::array<std::array<double, NC>, 3> x{};
            for (int c = 0; c < NC; ++c)
                zi[c] = z[c * n + i];
            for (int p = 0; p < 3; ++p)
                for (int c = 0; c < NC; ++c)
                    x[p][c] = comps[(p * NC + c) * n + i];
            try
            {
                const auto r = flash.stabilityTest(
                    P[i], T[i], zi, PhasePresence(active[i]), x);
                stable[i] = r.stable;
                valid[i] = r.valid;
                uint8_t m = 0;
                for (int p = 0; p < 3; ++p)
                {
                    if (r.missingPhaseUnstable[p]) m |= uint8_t(1u << p);
                    if (trialSum) trialSum[p * n + i] = r.trialSum[p];
                    if (incipient)
                        for (int c = 0; c < NC; ++c)
                            incipient[(p * NC + c) * n + i] = r.incipientComposition[p][c];
                }
                unstableMask[i] = m;
            }
            catch (const std::exception &)
            {
                stable[i] = 0;
                valid[i] = 0;
                unstableMask[i] = 0xff;
            }
        }
    });
    return 0;
}

// -------------------------------------------------------------- natural ----
struct NaturalBase
{
    virtual ~NaturalBase() = default;
    virtual int initPtz(const double *P, const double *z, double *primary, double *ps) = 0;
    virtual int setHistory(const double *primary, const double *ps) = 0;
    virtual int updateState(double *primary, double *ps, nz_report *report) = 0;
    virtual void setThreads(int n) = 0;
    // Seconds each cell's updatePhaseState took in the last updateState.
    std::vector<double> cellSeconds;
    virtual int residual(const double *primary, const double *ps, double *F) = 0;
    virtual int jacobian(const double *primary, const double *ps, double *vals) = 0;
    virtual int pattern(int64_t *rowPtr, int64_t *colIdx, int64_t *nnzb) = 0;
    virtual int accumulation(double *out) = 0;
};

template <int NC>
struct Natural final : NaturalBase
{
    using I = AIdx<NC>;
    using Eval = typename I::ValueType;
    static constexpr int B = I::numPrimaryVariables;
    static constexpr int NPS = I::numPhaseStateVariables;
    using Kernel = NaturalCellKernel<I>;
    using PrimaryArray = typename Kernel::PrimaryArray;
    using State = typename Kernel::State;
    using Props = typename Kernel::Properties;
    using Codec = PetscPhaseStateCodec<I>;

    std::unique_ptr<FluidSystem<I>> fluid;
    std::unique_ptr<Kernel> kernel;
    // Worker threads of the cell loops, one kernel each (the flash inside a
    // kernel keeps a mutable parameter cache, three_phase_flash.hpp:598).
    int threads{1};
    std::vector<std::unique_ptr<Kernel>> workers;

    void setThreads(int n) override
    {
        threads = n < 1 ? 1 : n;
        workers.resize(static_cast<std::size_t>(threads));
        for (int t = 1; t < threads; ++t)
            if (!workers[t])
                workers[t] = std::make_unique<Kernel>(*fluid);
    }
    const Kernel &worker(int t) const { return t == 0 ? *kernel : *workers[static_cast<std::size_t>(t)]; }
    int64_t ncell{0};
    std::vector<double> porosity, volume, trans, grav;
    std::vector<int64_t> offset, neighbor;
    double dt{1.0}, fscale{1.0};
    std::vector<AccumulationResult<I, double>> previousAccumulation;
    std::vector<CellProperties<I, double>> previousProperties;
    // BAIJ pattern (rows sorted) and the slot of each directed connection.
    std::vector<int64_t> rowPtr, colIdx, selfSlot, connSlot;

    Natural(const nz_fluid_desc &d, const nz_natural_desc &n)
    {
        typename FluidSystem<I>::PhaseArray surface{730.0, 1.8, 985.4};
        typename FluidSystem<I>::PhaseArray visc{2.4e-4, 1.86e-5, 4.69e-4};
        typename FluidSystem<I>::ComponentNames names{};
        for (int c = 0; c < NC; ++c)
            names[c] = "c" + std::to_string(c);
        fluid = std::make_unique<FluidSystem<I>>(
            surface, visc, makeEos<I>(d, d.sw_salinity), names,
            typename FluidSystem<I>::PhaseNames{"Oil", "Gas", "Water"},
            n.temperature);
        fluid->configureFullyCompositionalThreePhase(d.water_component);
        const nz_relperm_desc rp = n.relperm;
        // The quadratic curves of case/h2o_co2_nc10_2d_benchmark/benchmark_common.hpp:97-126.
        fluid->waterRelativePermeability = [rp](Eval sw) {
            const double v = scalarValue(sw);
            if (v <= rp.swc) return Eval(0.0);
            if (v >= 1.0 - rp.sorw) return Eval(rp.krw_max);
            const Eval se = (sw - rp.swc) / (1.0 - rp.swc - rp.sorw);
            return Eval(rp.krw_max) * se * se;
        };
        fluid->gasRelativePermeability = [rp](Eval sg) {
            const double v = scalarValue(sg);
            if (v <= rp.sgc) return Eval(0.0);
            if (v >= 1.0 - rp.sorg - rp.swc) return Eval(rp.krg_max);
            const Eval se = (sg - rp.sgc) / (1.0 - rp.sorg - rp.swc - rp.sgc);
            return Eval(rp.krg_max) * se * se;
        };
        fluid->threePhaseOilRelativePermeability = [rp](Eval, Eval so, Eval) {
            const double v = scalarValue(so);
            if (v <= rp.sorg) return Eval(0.0);
            if (v >= 1.0 - rp.swc) return Eval(rp.kro_max);
            const Eval se = (so - rp.sorg) / (1.0 - rp.swc - rp.sorg);
            return Eval(rp.kro_max) * se * se;
        };
        kernel = std::make_unique<Kernel>(*fluid);
        ncell = n.ncell;
        porosity.assign(n.porosity, n.porosity + ncell);
        volume.assign(n.volume, n.volume + ncell);
        offset.assign(n.conn_offset, n.conn_offset + ncell + 1);
        const int64_t nconn = offset.back();
        neighbor.assign(n.conn_neighbor, n.conn_neighbor + nconn);
        trans.assign(n.conn_trans, n.conn_trans + nconn);
        grav.assign(n.conn_gravity, n.conn_gravity + nconn);
        dt = n.time_step;
        fscale = n.fugacity_scaling;
        buildPattern();
    }

    void buildPattern()
    {
        // rows: self + every face neighbour (jacobian_factory.hpp:39-245, no wells)
        std::vector<std::vector<int64_t>> cols(static_cast<std::size_t>(ncell));
        for (int64_t c = 0; c < ncell; ++c)
        {
            cols[c].push_back(c);
            for (int64_t k = offset[c]; k < offset[c + 1]; ++k)
                cols[c].push_back(neighbor[k]);
            std::sort(cols[c].begin(), cols[c].end());
            cols[c].erase(std::unique(cols[c].begin(), cols[c].end()), cols[c].end());
        }
        rowPtr.assign(ncell + 1, 0);
        for (int64_t c = 0; c < ncell; ++c)
            rowPtr[c + 1] = rowPtr[c] + static_cast<int64_t>(cols[c].size());
        colIdx.resize(rowPtr.back());
        for (int64_t c = 0; c < ncell; ++c)
            std::copy(cols[c].begin(), cols[c].end(), colIdx.begin() + rowPtr[c]);
        auto slot = [&](int64_t row, int64_t col) {
            const auto b = colIdx.begin() + rowPtr[row];
            const auto e = colIdx.begin() + rowPtr[row + 1];
            return static_cast<int64_t>(std::lower_bound(b, e, col) - colIdx.begin());
        };
        selfSlot.resize(ncell);
        connSlot.resize(neighbor.size());
        for (int64_t c = 0; c < ncell; ++c)
        {
            selfSlot[c] = slot(c, c);
            for (int64_t k = offset[c]; k < offset[c + 1]; ++k)
                connSlot[k] = slot(neighbor[k], c);
        }
    }

    int pattern(int64_t *rp, int64_t *ci, int64_t *nnzb) override
    {
        if (nnzb) *nnzb = rowPtr.back();
        if (rp) std::copy(rowPtr.begin(), rowPtr.end(), rp);
        if (ci) std::copy(colIdx.begin(), colIdx.end(), ci);
        return 0;
    }

    static PrimaryArray readPrimary(const double *x, int64_t c)
    {
        PrimaryArray a{};
        for (int k = 0; k < B; ++k)
            a[k] = x[c * B + k];
        return a;
    }
    static PhaseStateData<I> readPs(const double *ps, int64_t c)
    {
        typename Codec::Array a{};
        for (int k = 0; k < NPS; ++k)
            a[k] = ps[c * NPS + k];
        return Codec::decode(a);
    }
    static void writePrimary(double *x, int64_t c, const PrimaryArray &a)
    {
        for (int k = 0; k < B; ++k)
            x[c * B + k] = a[k];
    }
    static void writePs(double *ps, int64_t c, const PhaseStateData<I> &s)
    {
        const auto a = Codec::encode(s);
        for (int k = 0; k < NPS; ++k)
            ps[c * NPS + k] = a[k];
    }

    int initPtz(const double *P, const double *z, double *primary, double *ps) override
    {
        for (int64_t c = 0; c < ncell; ++c)
        {
            std::array<double, NC> zc{};
            for (int i = 0; i < NC; ++i)
                zc[i] = z[c * NC + i];
            const auto flash = kernel->phaseEquilibrium().flashPTZ(
                P[c], fluid->temperature, zc);
            if (!flash.converged)
                return static_cast<int>(c + 1);
            PrimaryArray a{};
            a[I::Primary::pressure] = P[c];
            PhaseStateData<I> s;
            kernel->phaseEquilibrium().assignFlashResult(a, s, flash);
            writePrimary(primary, c, a);
            writePs(ps, c, s);
        }
        return 0;
    }

    struct CacheEntry
    {
        State state;
        Props props;
    };

    std::vector<CacheEntry> buildCache(const double *primary, const double *ps) const
    {
        // buildCellCache_ (natural_petsc_runtime_cell_cache.inc:66-116)
        std::vector<CacheEntry> cache(static_cast<std::size_t>(ncell));
        parallelFor(ncell, threads, [&](int64_t b, int64_t e, int t) {
            const Kernel &k = worker(t);
            for (int64_t c = b; c < e; ++c)
            {
                const auto a = readPrimary(primary, c);
                const auto s = readPs(ps, c);
                cache[c].state = k.decodeState(a, s);
                typename Kernel::Composition overall{};
                for (int i = 0; i < NC; ++i)
                    overall[i] = Eval(s.overallComposition[i]);
                cache[c].props = k.evaluateProperties(cache[c].state, Eval(porosity[c]), 0.0, 2.0, &overall);
            }
        });
        return cache;
    }

    int setHistory(const double *primary, const double *ps) override
    {
        const auto cache = buildCache(primary, ps);
        previousProperties.resize(ncell);
        previousAccumulation.resize(ncell);
        for (int64_t c = 0; c < ncell; ++c)
        {
            previousProperties[c] = scalarizeCellProperties<I>(cache[c].props);
            previousAccumulation[c] = computeFluidAccumulation<I>(previousProperties[c], -1);
        }
        return 0;
    }

    int accumulation(double *out) override
    {
        for (int64_t c = 0; c < ncell; ++c)
            for (int i = 0; i < NC; ++i)
                out[c * NC + i] = previousAccumulation[c].componentMass[i];
        return 0;
    }

    int updateState(double *primary, double *ps, nz_report *report) override
    {
        cellSeconds.assign(static_cast<std::size_t>(ncell), 0.0);
        std::vector<PrimaryArray> newPrimary(ncell);
        std::vector<PhaseStateData<I>> newPs(ncell);
        nz_report r{};
        r.succeeded = 1;
        r.first_failure_cell = -1;
        // every cell's update (independent), then the transaction in cell order
        std::vector<PhaseUpdateResult> results(static_cast<std::size_t>(ncell));
        parallelFor(ncell, threads, [&](int64_t b, int64_t e, int t) {
            const auto &eq = worker(t).phaseEquilibrium();
            for (int64_t c = b; c < e; ++c)
            {
                auto a = readPrimary(primary, c);
                auto s = readPs(ps, c);
                const auto t0 = std::chrono::steady_clock::now();
                eq.sanitizePrimaryBeforeFlash(a, false);
                PhaseUpdateResult u;
                try
                {
                    u = eq.updatePhaseState(a, s);
                }
                catch (const std::exception &)
                {
                    u.status = PhaseUpdateStatus::RecoverableThermodynamicFailure;
                }
                cellSeconds[c] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                results[c] = u;
                newPrimary[c] = a;
                newPs[c] = s;
            }
        });
        for (int64_t c = 0; c < ncell; ++c)
        {
            const PhaseUpdateResult &u = results[c];
            if (u.recoverableFailure())
            {
                r.succeeded = 0;
                r.first_failure_cell = c;
                r.status = static_cast<int32_t>(u.status);
                r.phase_removed = u.phaseRemoved;
                r.missing_phase_unstable = u.missingPhaseUnstable;
                r.stability_invalid = u.stabilityInvalid;
                r.restricted_flash_failed = u.restrictedFlashFailed;
                r.unrestricted_flash_failed = u.unrestrictedFlashFailed;
                r.failed_cells = 1;
                break;
            }
            ++r.updated_cells;
            if (u.status == PhaseUpdateStatus::StableReducedSet)
                ++r.stable_reduced_cells;
        }
        if (report) *report = r;
        if (!r.succeeded)
            return 1;
        for (int64_t c = 0; c < ncell; ++c)
        {
            writePrimary(primary, c, newPrimary[c]);
            writePs(ps, c, newPs[c]);
        }
        return 0;
    }

    int residual(const double *primary, const double *ps, double *F) override
    {
        if (previousAccumulation.size() != static_cast<std::size_t>(ncell))
            return -1;
        const auto cache = buildCache(primary, ps);
        parallelFor(ncell, threads, [&](int64_t b, int64_t e, int t) {
        const Kernel &k = worker(t);
        for (int64_t c = b; c < e; ++c)
        {
            FaceMassFlux<I, double> outward{};
            for (int64_t k = offset[c]; k < offset[c + 1]; ++k)
            {
                const int64_t nb = neighbor[k];
                const auto flux = computeFaceMassFluxValue<I, Eval>(
                    cache[c].state, cache[c].props, cache[nb].state, cache[nb].props,
                    trans[k], grav[k], volume[c], volume[nb], c, nb, -1, nullptr);
                for (int i = 0; i < NC; ++i)
                    outward.component[i] += flux.component[i];
            }
            auto block = k.assembleLocalResidual(
                cache[c].state, cache[c].props, previousProperties[c], volume[c], dt,
                fscale, -1, 2650.0, nullptr, &previousAccumulation[c], nullptr);
            std::array<Eval, NC> zeroSource{};
            addCellConservationTransportAndWell<I>(block, outward, zeroSource, Eval(0.0));
            for (int q = 0; q < B; ++q)
                F[c * B + q] = block.value[q].value();
        }
        });
        return 0;
    }

    int jacobian(const double *primary, const double *ps, double *vals) override
    {
        if (previousAccumulation.size() != static_cast<std::size_t>(ncell))
            return -1;
        const auto cache = buildCache(primary, ps);
        std::fill(vals, vals + rowPtr.back() * B * B, 0.0);
        parallelFor(ncell, threads, [&](int64_t b, int64_t e, int t) {
        const Kernel &k = worker(t);
        for (int64_t c = b; c < e; ++c)
        {
            const auto block = k.assembleLocalResidual(
                cache[c].state, cache[c].props, previousProperties[c], volume[c], dt,
                fscale, -1, 2650.0, nullptr, &previousAccumulation[c], nullptr);
            double *self = vals + selfSlot[c] * B * B;
            for (int row = 0; row < B; ++row)
                for (int col = 0; col < B; ++col)
                    self[row * B + col] = block.value[row].derivative(col);
            for (int64_t k = offset[c]; k < offset[c + 1]; ++k)
            {
                const int64_t nb = neighbor[k];
                const auto flux = computeFaceMassFlux<I, Eval>(
                    cache[c].state, cache[c].props, cache[nb].state, cache[nb].props,
                    trans[k], grav[k], volume[c], volume[nb], c, nb, -1, nullptr);
                double *recip = vals + connSlot[k] * B * B;
                for (int i = 0; i < NC; ++i)
                {
                    const int row = I::Equation::massConservation[i];
                    for (int col = 0; col < B; ++col)
                    {
                        const double dv = flux.component[i].derivative(col);
                        self[row * B + col] += dv;
                        recip[row * B + col] = -dv;
                    }
                }
            }
        }
        });
        return 0;
    }
};

template <template <int> class F, class... Args>
int dispatchNc(int nc, Args &&...args)
{
    switch (nc)
    {
    case 2: return F<2>::run(std::forward<Args>(args)...);
    case 3: return F<3>::run(std::forward<Args>(args)...);
    case 4: return F<4>::run(std::forward<Args>(args)...);
    case 5: return F<5>::run(std::forward<Args>(args)...);
    case 6: return F<6>::run(std::forward<Args>(args)...);
    case 8: return F<8>::run(std::forward<Args>(args)...);
    default: g_error = "oracle: unsupported nc"; return NZ_ERR_UNSUPPORTED;
    }
}

// ---- boundary distance of a converged flash answer (|TPD| of its missing
// phases).  stabilityTest reports the largest trial sum of each missing phase,
// which is exactly 1 whenever a trial falls back onto an existing phase (a
// trivial stationary point), so it cannot say how far a point is from the
// boundary.  This restates stabilityTest's trial loop
// (three_phase_flash.hpp:399-480) with the reference's own seed list and
// trial solver, keeping only the non-trivial trials that do not coincide with
// an active phase: distance = min over missing phases of |1 - best such sum|
// (infinite when no such stationary point exists).  The private members are
// reached through the standard explicit-instantiation access rule.
template <int NC>
struct TrialAccess
{
    friend auto trialFn(TrialAccess<NC>);
    friend auto seedsFn(TrialAccess<NC>);
    friend auto phaseFn(TrialAccess<NC>);
};
template <int NC, auto Trial, auto Seeds, auto Phase>
struct TrialRob
{
    friend auto trialFn(TrialAccess<NC>) { return Trial; }
    friend auto seedsFn(TrialAccess<NC>) { return Seeds; }
    friend auto phaseFn(TrialAccess<NC>) { return Phase; }
};
#define NZ_TRIAL_ROB(NCV)                                                                              \
    template struct TrialRob<NCV, &CubicThreePhaseFlash<SIdx<NCV>>::stabilityTrial_,                  \
                             &CubicThreePhaseFlash<SIdx<NCV>>::stabilitySeeds_,                      \
                             &CubicThreePhaseFlash<SIdx<NCV>>::phaseResult_>;
NZ_TRIAL_ROB(2)
NZ_TRIAL_ROB(3)
NZ_TRIAL_ROB(4)
NZ_TRIAL_ROB(5)
NZ_TRIAL_ROB(6)
NZ_TRIAL_ROB(8)
#undef NZ_TRIAL_ROB

template <int NC>
int boundaryBatch(const nz_fluid_desc *d, const nz_flash_options *o, int64_t n, const double *P,
                  const double *T, const double *z, const double *salinity, const uint8_t *presence,
                  const double *comps, double *distance, int threads)
{
    using I = SIdx<NC>;
    using Flash = CubicThreePhaseFlash<I>;
    const auto options = toOptions(o, d->water_component);
    const auto trialOf = trialFn(TrialAccess<NC>{});
    const auto seedsOf = seedsFn(TrialAccess<NC>{});
    const auto phaseOf = phaseFn(TrialAccess<NC>{});
    const CompositionalPhase phases[3] = {CompositionalPhase::Oil, CompositionalPhase::Gas,
                                          CompositionalPhase::Water};
    parallelFor(n, threads, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i)
        {
            distance[i] = std::numeric_limits<double>::infinity();
            const uint8_t active = presence[i];
            if (active == 0 || active == 7)
                continue;
            const auto eos = makeEos<I>(*d, salinity ? salinity[i] : d->sw_salinity);
            Flash flash(eos, options);
            std::array<double, NC> zi{};
            std::array<std::array<double, NC>, 3> x{};
            double zs = 0.0;
            for (int c = 0; c < NC; ++c)
                zs += (zi[c] = z[c * n + i]);
            for (int c = 0; c < NC; ++c)
                zi[c] /= zs;
            for (int p = 0; p < 3; ++p)
            {
                double s = 0.0;
                for (int c = 0; c < NC; ++c)
                    s += (x[p][c] = comps[(p * NC + c) * n + i]);
                if (active & (1u << p))
                    for (int c = 0; c < NC; ++c)
                        x[p][c] /= s;
            }
            int ref = 0;
            while (!(active & (1u << ref)))
                ++ref;
            try
            {
                const auto refThermo = (flash.*phaseOf)(phases[ref], P[i], T[i], x[ref]);
                std::array<double, NC> logReference{};
                for (int c = 0; c < NC; ++c)
                    logReference[c] = std::log(std::max(x[ref][c], options.compositionFloor)) +
                                      std::log(std::max(refThermo.fugacityCoefficient[c], 1.0e-300));
                const double coincidence = std::max(10.0 * options.coincidentPhaseCompositionTolerance, 1.0e-7);
                double dist = std::numeric_limits<double>::infinity();
                for (int p = 0; p < 3; ++p)
                {
                    if (active & (1u << p))
                        continue;
                    const auto seeds = (flash.*seedsOf)(phases[p], P[i], T[i], zi, x[ref]);
                    for (std::size_t k = 0; k < seeds.size; ++k)
                    {
                        const auto t = (flash.*trialOf)(phases[p], P[i], T[i], logReference, x[ref], seeds.values[k]);
                        if (!t.valid || t.trivial)
                            continue;
                        bool coincides = false;
                        for (int q = 0; q < 3 && !coincides; ++q)
                        {
                            if (!(active & (1u << q)))
                                continue;
                            double m = 0.0;
                            for (int c = 0; c < NC; ++c)
                                m = std::max(m, std::abs(t.composition[c] - x[q][c]));
                            coincides = m <= coincidence;
                        }
                        if (!coincides)
                            dist = std::min(dist, std::abs(1.0 - t.sum));
                    }
                }
                distance[i] = dist;
            }
            catch (const std::exception &)
            {
                distance[i] = std::numeric_limits<double>::quiet_NaN();
            }
        }
    });
    return NZ_OK;
}

template <int NC> struct FlashRun { template <class... A> static int run(A &&...a) { return flashBatch<NC>(std::forward<A>(a)...); } };
template <int NC> struct EosRun { template <class... A> static int run(A &&...a) { return eosBatch<NC>(std::forward<A>(a)...); } };
template <int NC> struct StabRun { template <class... A> static int run(A &&...a) { return stabilityBatch<NC>(std::forward<A>(a)...); } };
template <int NC> struct BoundaryRun { template <class... A> static int run(A &&...a) { return boundaryBatch<NC>(std::forward<A>(a)...); } };

template <class F>
int guarded(F &&f)
{
    try
    {
        return f();
    }
    catch (const std::exception &ex)
    {
        g_error = ex.what();
        return NZ_ERR_ARGUMENT;
    }
}
} // namespace

extern "C" {

const char *nzref_last_error(void) { return g_error.c_str(); }

int nzref_flash_batch(const nz_fluid_desc *d, const nz_flash_options *o, int64_t n,
                      const double *P, const double *T, const double *z,
                      const double *salinity, const nz_flash_out *out, int threads)
{
    return guarded([&] { return dispatchNc<FlashRun>(d->nc, d, o, n, P, T, z, salinity, out, threads); });
}

int nzref_eos_phase_batch(const nz_fluid_desc *d, int64_t n, const double *P,
                          const double *T, const double *x, const int8_t *role,
                          const double *salinity, double *Z, double *lnphi)
{
    return guarded([&] { return dispatchNc<EosRun>(d->nc, d, n, P, T, x, role, salinity, Z, lnphi); });
}

int nzref_stability_batch(const nz_fluid_desc *d, const nz_flash_options *o, int64_t n,
                          const double *P, const double *T, const double *z,
                          const double *salinity, const uint8_t *active,
                          const double *comps, uint8_t *stable, uint8_t *valid,
                          uint8_t *unstableMask, double *trialSum, double *incipient,
                          int threads)
{
    return guarded([&] {
        return dispatchNc<StabRun>(d->nc, d, o, n, P, T, z, salinity, active, comps,
                                   stable, valid, unstableMask, trialSum, incipient, threads);
    });
}

int nzref_boundary_distance(const nz_fluid_desc *d, const nz_flash_options *o, int64_t n,
                            const double *P, const double *T, const double *z,
                            const double *salinity, const uint8_t *presence,
                            const double *comps, double *distance, int threads)
{
    return guarded([&] {
        return dispatchNc<BoundaryRun>(d->nc, d, o, n, P, T, z, salinity, presence, comps, distance, threads);
    });
}

void *nzref_natural_create(const nz_fluid_desc *d, const nz_natural_desc *n)
{
    try
    {
        switch (d->nc)
        {
        case 3: return new Natural<3>(*d, *n);
        case 4: return new Natural<4>(*d, *n);
        case 5: return new Natural<5>(*d, *n);
        case 6: return new Natural<6>(*d, *n);
        case 8: return new Natural<8>(*d, *n);
        default: g_error = "oracle: unsupported nc"; return nullptr;
        }
    }
    catch (const std::exception &ex)
    {
        g_error = ex.what();
        return nullptr;
    }
}

void nzref_natural_destroy(void *h) { delete static_cast<NaturalBase *>(h); }

int nzref_natural_init_ptz(void *h, const double *P, const double *z, double *primary, double *ps)
{
    return guarded([&] { return static_cast<NaturalBase *>(h)->initPtz(P, z, primary, ps); });
}
int nzref_natural_set_history(void *h, const double *primary, const double *ps)
{
    return guarded([&] { return static_cast<NaturalBase *>(h)->setHistory(primary, ps); });
}
int nzref_natural_accumulation(void *h, double *out)
{
    return guarded([&] { return static_cast<NaturalBase *>(h)->accumulation(out); });
}
int nzref_update_state(void *h, double *primary, double *ps, nz_report *report)
{
    return guarded([&] { return static_cast<NaturalBase *>(h)->updateState(primary, ps, report); });
}
int nzref_residual(void *h, const double *primary, const double *ps, double *F)
{
    return guarded([&] { return static_cast<NaturalBase *>(h)->residual(primary, ps, F); });
}
int nzref_jacobian(void *h, const double *primary, const double *ps, double *vals)
{
    return guarded([&] { return static_cast<NaturalBase *>(h)->jacobian(primary, ps, vals); });
}
void nzref_natural_set_threads(void *h, int threads)
{
    static_cast<NaturalBase *>(h)->setThreads(threads);
}
// Per-cell seconds of the last update (out: ncell doubles); returns the count.
int64_t nzref_natural_update_cell_seconds(void *h, double *out)
{
    const auto &v = static_cast<NaturalBase *>(h)->cellSeconds;
    for (std::size_t c = 0; c < v.size(); ++c)
        out[c] = v[c];
    return int64_t(v.size());
}
int nzref_natural_pattern(void *h, int64_t *rowPtr, int64_t *colIdx, int64_t *nnzb)
{
    return guarded([&] { return static_cast<NaturalBase *>(h)->pattern(rowPtr, colIdx, nnzb); });
}

} // extern "C"
