/*
 * nonenone_b200.h -- C ABI of the B200 (sm_100a) thermodynamics + Natural
 * assembly hot path of the MPMC_SCW reservoir simulator.
 *
 * Every entry point takes plain pointers and sizes; no C++ or CUDA types
 * cross this boundary (streams are passed as `void*` = cudaStream_t).
 * Return codes: 0 = success, > 0 = recoverable (the host treats it like the
 * reference's thermodynamic failure / SNESSetFunctionDomainError),
 * < 0 = fatal (bad argument, CUDA error).  The message of the last failing
 * call on the calling host thread is available from nz_last_error().
 *
 * Reference interfaces replaced (paths inside the MPMC_SCW tree):
 *   nz_eos_phase_batch   CubicEquationOfState::phaseResult
 *                        (models/include/natural/thermo/cubic_eos.hpp:806-857)
 *   nz_flash_batch       CubicThreePhaseFlash::flash
 *                        (models/include/natural/thermo/three_phase_flash.hpp:83-227)
 *   nz_stability_batch   CubicThreePhaseFlash::stabilityTest
 *                        (three_phase_flash.hpp:300-489)
 *   nz_update_state      NaturalPetscRuntime::updateStateWithReport
 *                        (models/include/natural/petsc/detail/natural_petsc_runtime_state.inc:166-345)
 *   nz_residual          NaturalPetscRuntime::formFunction
 *                        (natural_petsc_runtime_residual.inc:19-133)
 *   nz_jacobian          NaturalPetscRuntime::assembleJacobian_
 *                        (natural_petsc_runtime_jacobian.inc:8-109,120-299)
 *   nz_jacobian_columns  the same, in the per-cell column order of its
 *                        MatSetValuesBlocked calls (jacobian.inc:279-299)
 *   nz_natural_init_ptz  NaturalPetscRuntime::initializeUniformFromPTZ
 *                        (natural_petsc_runtime_state.inc:107-164), per cell
 *   nz_natural_pattern   buildNaturalJacobianPattern
 *                        (models/include/natural/petsc/jacobian_factory.hpp:39-245)
 */
#ifndef NONENONE_B200_H
#define NONENONE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NZ_ABI_VERSION 2
#define NZ_MAX_NC 8

/* ---- status codes ------------------------------------------------------ */
#define NZ_OK 0
#define NZ_RECOVERABLE 1          /* thermodynamic failure, state rolled back */
#define NZ_ERR_ARGUMENT (-1)
#define NZ_ERR_CUDA (-2)
#define NZ_ERR_UNSUPPORTED (-3)
#define NZ_ERR_ALLOC (-4)
#define NZ_ERR_SELFCHECK (-5)     /* a device self-check (queue bound, spin guard) stopped a batch */

/* per-point flash status (nz_flash_out.status) */
#define NZ_FLASH_CONVERGED 0
#define NZ_FLASH_FAILED 1          /* every path failed; same as reference converged=false */
#define NZ_FLASH_BAD_INPUT 2       /* non-finite or non-positive P, T or z (reference throws) */
#define NZ_FLASH_EOS_ERROR 3       /* no admissible cubic root etc. (reference throws) */
#define NZ_FLASH_NOT_PORTED 4      /* reached a fail-only recovery this build does not carry */
#define NZ_FLASH_UNFINISHED 5      /* a device self-check of the staged batch stopped before this
                                      point was done (see nz_flash_check); no reference counterpart */

/* ---- fluid description --------------------------------------------------
 * Mirrors CompositionalMixture + CubicEquationOfState configuration
 * (compositional_mixture.hpp, cubic_eos.hpp:170-192, soreide_whitson.hpp).
 */
#define NZ_EOS_PR 0
#define NZ_EOS_SW 1
#define NZ_EOS_CPA 2

/* CPA cubic term and radial distribution (thermodynamic_model.hpp:19-23,
 * cubic_plus_association.hpp:19-23) */
#define NZ_CPA_SRK 0
#define NZ_CPA_PR 1
#define NZ_CPA_RADIAL_SIMPLIFIED 0
#define NZ_CPA_RADIAL_CARNAHAN_STARLING 1

/* SW aqueous H2O-solute BIP correlation per component (cubic_eos.hpp:2389-2404) */
#define NZ_SW_BIP_KIJ 0            /* keep the ordinary k_ij */
#define NZ_SW_BIP_CONSTANT 1       /* sw_bip_value[c] */
#define NZ_SW_BIP_CO2 2            /* SoreideWhitsonCorrelations::co2AqueousBip */
#define NZ_SW_BIP_HYDROCARBON 3    /* SoreideWhitsonCorrelations::hydrocarbonAqueousBip */
#define NZ_SW_BIP_CO2_CHABAB 4     /* SoreideWhitsonCorrelations::co2AqueousBipChabab2019 */

typedef struct nz_fluid_desc {
    int32_t nc;                 /* components, 2..NZ_MAX_NC */
    int32_t eos_model;          /* NZ_EOS_* */
    int32_t eos_type;           /* 1 = PR, 5 = PR78 m(omega) when omega > 0.49 */
    int32_t water_component;    /* H2O index, -1 = none */
    double omega_a, omega_b;    /* 0.4572355, 0.0779691 */
    double m1, m2;              /* 1 +/- sqrt(2) */
    double minimum_composition; /* EOS-level RR floor (cubic_eos.hpp:185) */
    double tc[NZ_MAX_NC];       /* K */
    double pc[NZ_MAX_NC];       /* Pa */
    double vc[NZ_MAX_NC];       /* m3/mol */
    double acentric[NZ_MAX_NC];
    double mw[NZ_MAX_NC];       /* kg/mol */
    double kij[NZ_MAX_NC * NZ_MAX_NC];
    double sw_salinity;         /* NaCl molality used when no per-point salinity */
    int32_t sw_bip_kind[NZ_MAX_NC];
    double sw_bip_value[NZ_MAX_NC];
    /* PR-CPA / SRK-CPA (eos_model = NZ_EOS_CPA): CubicEquationOfState::
     * CubicPlusAssociationOptions (models/include/natural/thermo/cubic_eos.hpp:117-136).
     * The flash and EOS entry points carry one associating component with equal
     * donor and acceptor sites, or one donor-bearing component with any acceptors
     * (e.g. 4C water with CO2 as an acceptor); fluids with several donor-bearing
     * components give NZ_FLASH_NOT_PORTED per point, and nz_natural_create
     * refuses them. */
    double cpa_a0[NZ_MAX_NC];            /* Pa m6/mol2 */
    double cpa_b[NZ_MAX_NC];             /* m3/mol */
    double cpa_c1[NZ_MAX_NC];
    double cpa_epsilon[NZ_MAX_NC];       /* association energy, J/mol */
    double cpa_beta[NZ_MAX_NC];          /* association volume */
    int32_t cpa_donor_sites[NZ_MAX_NC];
    int32_t cpa_acceptor_sites[NZ_MAX_NC];
    double cpa_cross_epsilon[NZ_MAX_NC * NZ_MAX_NC];  /* [donor][acceptor]; positive */
    double cpa_cross_beta[NZ_MAX_NC * NZ_MAX_NC];     /* entries override the CR-1 rule */
    int32_t cpa_physical_term;           /* NZ_CPA_SRK or NZ_CPA_PR */
    int32_t cpa_radial;                  /* NZ_CPA_RADIAL_SIMPLIFIED or _CARNAHAN_STARLING */
    int32_t cpa_max_association_iterations;  /* 2000 */
    double cpa_association_tolerance;    /* 1e-12 */
    double cpa_association_damping;      /* 0.2 */
} nz_fluid_desc;

/* ThreePhaseFlashOptions (three_phase_flash_types.hpp:21-41) */
typedef struct nz_flash_options {
    int32_t maximum_iterations;                 /* 120 */
    int32_t maximum_rachford_rice_iterations;   /* 80 */
    int32_t maximum_stability_iterations;       /* 80 */
    int32_t stability_ssi_before_newton;        /* 8 */
    int32_t maximum_stability_newton;           /* 12 */
    int32_t two_phase_ssi_before_newton;        /* 8 */
    int32_t maximum_two_phase_newton;           /* 12 */
    int32_t three_phase_ssi_before_newton;      /* 10 */
    int32_t maximum_three_phase_newton;         /* 12 */
    double fugacity_tolerance;                  /* 1e-9 */
    double rachford_rice_tolerance;             /* 1e-12 */
    double stability_tolerance;                 /* 1e-9 */
    double phase_fraction_tolerance;            /* 1e-10 */
    double coincident_composition_tolerance;    /* 1e-8 */
    double composition_floor;                   /* 1e-30 */
    double log_k_step_limit;                    /* 2 */
    double numerical_jacobian_step;             /* 1e-6 */
} nz_flash_options;

/* Fill *opts with the reference defaults. */
void nz_flash_options_default(nz_flash_options* opts);

/* ---- context -------------------------------------------------------------- */
typedef struct nz_ctx nz_ctx;

int nz_ctx_create(const nz_fluid_desc* fluid, const nz_flash_options* options,
                  int32_t device, nz_ctx** out);
int nz_ctx_destroy(nz_ctx* ctx);
const char* nz_last_error(void);
int32_t nz_abi_version(void);

/* ---- EOS phase evaluation ---------------------------------------------------
 * role[i]: 0 = Oil (liquid root), 1 = Gas (vapour root), 2 = Water (liquid
 * root, SW aqueous BIPs).  Outputs Z[n], lnphi[nc*n] (component-major SoA:
 * lnphi[c*n+i]).  Device pointers, stream ordered.
 * Replaces CubicEquationOfState::phaseResult(P,T,x,phase)
 * (cubic_eos.hpp:833-852).
 */
int nz_eos_phase_batch(nz_ctx* ctx, int64_t n, const double* pressure,
                       const double* temperature, const double* x,
                       const int8_t* role, const double* salinity,
                       double* compressibility, double* ln_phi,
                       void* stream);

/* ---- P-T-z flash ----------------------------------------------------------
 * Replaces CubicThreePhaseFlash::flash(P,T,z) for a batch
 * (three_phase_flash.hpp:83-227).  Inputs: pressure[n] Pa, temperature[n] K,
 * z[nc*n] (component-major), salinity[n] (SW only, NULL = sw_salinity).
 * Output arrays are phase-major SoA; any pointer may be NULL.
 */
typedef struct nz_flash_out {
    uint8_t* presence;        /* [n]  PhasePresence bits (1 oil, 2 gas, 4 water) */
    uint8_t* status;          /* [n]  NZ_FLASH_* */
    double* beta;             /* [3*n]       phaseMoleFraction[p] at p*n+i */
    double* saturation;       /* [3*n] */
    double* composition;      /* [3*nc*n]    x[p][c] at (p*nc+c)*n+i */
    double* compressibility;  /* [3*n] */
    double* molar_density;    /* [3*n] */
    double* k_gas_oil;        /* [nc*n] */
    double* k_water_oil;      /* [nc*n] */
    int32_t* iterations;      /* [n] */
} nz_flash_out;

#define NZ_PRECISION_FP64 0         /* plain FP64 form: one thread runs one point's whole flash */
#define NZ_PRECISION_MIXED 1        /* staged; leading SSI steps of the TPD trials with FP32 mixing and
                                       ln phi (FP64 root), every trial finished in FP64, and a final FP64
                                       ln-fugacity Newton polish of the multiphase answers to 1e-11 */
#define NZ_PRECISION_FP64_STAGED 2  /* staged, every TPD trial in FP64 exactly as the plain form */

int nz_flash_batch(nz_ctx* ctx, int64_t n, const double* pressure,
                   const double* temperature, const double* z,
                   const double* salinity, const nz_flash_out* out,
                   int32_t precision, void* stream);

/* Host-pointer convenience: copies in, runs, copies out, synchronises. */
int nz_flash_batch_host(nz_ctx* ctx, int64_t n, const double* pressure,
                        const double* temperature, const double* z,
                        const double* salinity, const nz_flash_out* out,
                        int32_t precision);

/* Number of single-phase EOS evaluations (mixing+root+ln phi) the last
 * nz_flash_batch on this context executed; read after a stream sync. */
int nz_flash_eos_eval_count(nz_ctx* ctx, uint64_t* count);

/* Self-checks of the last staged batch on this context (no counterpart in the
 * reference, which has no device queues).  The staged kernels bound every
 * queue they fill and cap every lane-refill loop; a tripped check sets a
 * code here (0 = none), the kernels after it leave the unfinished points
 * alone, and those points keep status NZ_FLASH_UNFINISHED.  Read after the
 * batch's stream has been synchronised.  nz_flash_batch_host makes this
 * check itself and returns NZ_ERR_SELFCHECK when a code is set. */
int nz_flash_check(nz_ctx* ctx, int32_t* bound_code, int32_t* guard_code);

/* Iterations a lane-refill loop of the staged kernels may run before it gives
 * up (default 2^26, far above any solve); >= 1.  Lowering it is how a caller
 * (or a test) makes the spin guard run out without faulting the GPU. */
int nz_ctx_set_spin_limit(nz_ctx* ctx, int64_t limit);

/* ---- P-T-z flash without allocation ------------------------------------------
 * No counterpart in the reference (it has no GPU code): an extra entry point
 * for callers that must not allocate device memory while they run -- hosts
 * whose device memory is pre-claimed by another allocator (a PETSc or
 * framework memory pool holding the GPU, so a cudaMalloc at call time can
 * fail or fragment their pool) and deployments that fix every device
 * allocation at load time.  It runs the staged batched flash
 * (NZ_PRECISION_FP64_STAGED or NZ_PRECISION_MIXED) with its work space in a
 * static device array of NZ_NOALLOC_SCRATCH_BYTES that every GPU which loads
 * this library holds until the process exits; it calls no cudaMalloc /
 * cudaFree.  Batches whose work space would exceed the array are rejected
 * with NZ_ERR_ARGUMENT.  The limit depends on the fluid (its component count,
 * whether it has a water component, which adds a stability seed, and whether
 * it is Soreide-Whitson, which adds the allocation-search memos); the error
 * message states the exact limit for the context's fluid.  For PR / PR-CPA
 * fluids with a water component it is 13,980 points for nc = 3, 7,712 for
 * nc = 6 and 5,696 for nc = 8; for Soreide-Whitson fluids 10,808 / 6,047 /
 * 4,480.  The first call on a
 * device looks the array's device address up (cudaGetSymbolAddress) and
 * should therefore come before any stream capture.  All calls share the one
 * array and the context's evaluation counter: calls that overlap on the GPU
 * (other streams, other contexts) race and must be serialised by the caller.
 * Device pointers, stream ordered, same outputs as nz_flash_batch.
 */
#define NZ_NOALLOC_SCRATCH_BYTES (32ull << 20)
int nz_flash_batch_noalloc(nz_ctx* ctx, int64_t n, const double* pressure,
                           const double* temperature, const double* z,
                           const double* salinity, const nz_flash_out* out,
                           int32_t precision, void* stream);

/* ---- uneven multi-model batches -------------------------------------------
 * A host running many independent models (a fluid and its cells each) calls
 * CubicThreePhaseFlash::flash (three_phase_flash.hpp:83-227) per cell of each
 * model; on the device that is one nz_flash_batch per model.  nz_models runs
 * them together: the models of one component count share one staged launch
 * sequence (each point reads its model's fluid from a device table, so PR, SW
 * and PR-CPA models mix in the same kernels), the component-count groups run
 * on forked streams, and the whole call -- upload of the callers' pointers,
 * gather into group buffers, the staged kernels, scatter back -- is captured
 * once into a CUDA graph and replayed on every later call.  Each model's
 * answers are those of nz_flash_batch on that model alone.
 *
 * Point counts are fixed at creation (they size the group buffers and the
 * graph).  Precision: NZ_PRECISION_FP64_STAGED or NZ_PRECISION_MIXED.
 * Not thread safe; calls on one object are serialised by the caller.
 */
typedef struct nz_models nz_models;

typedef struct nz_model_io {
    const double* pressure;      /* [n] device */
    const double* temperature;   /* [n] device */
    const double* z;             /* [nc*n] device, component-major */
    const double* salinity;      /* [n] device, or NULL: the fluid's sw_salinity */
    nz_flash_out out;            /* the model's outputs (NULL fields are skipped) */
} nz_model_io;

/* options: NULL (defaults) or one per model. */
int nz_models_create(int32_t nmodels, const nz_fluid_desc* fluids,
                     const nz_flash_options* options, const int64_t* points,
                     int32_t device, nz_models** out);
int nz_models_destroy(nz_models* m);
int nz_models_flash(nz_models* m, const nz_model_io* io, int32_t precision, void* stream);
/* The autotuner: for every component count present, time the group's staged
 * sequence on a strided sample of its points (up to sample_points) for each
 * candidate launch shape and keep the fastest; the groups are timed side by
 * side on their own streams, as they run in the graph (the next
 * nz_models_flash captures a new graph).  Synchronises the stream. */
int nz_models_tune(nz_models* m, const nz_model_io* io, int32_t precision,
                   int64_t sample_points, void* stream);
/* Launch shape of a component count: resident blocks per SM of the lane
 * kernels and of the warp-per-point kernels. */
int nz_models_get_tuning(nz_models* m, int32_t nc, int32_t* lane_blocks_per_sm,
                         int32_t* warp_blocks_per_sm);
int nz_models_set_tuning(nz_models* m, int32_t nc, int32_t lane_blocks_per_sm,
                         int32_t warp_blocks_per_sm);
/* Self-check words of the last call (largest code over the groups). */
int nz_models_check(nz_models* m, int32_t* bound_code, int32_t* guard_code);
/* EOS evaluations of the last call (read after a stream sync). */
int nz_models_eos_eval_count(nz_models* m, uint64_t* count);

/* ---- tangent-plane stability ----------------------------------------------
 * Replaces CubicThreePhaseFlash::stabilityTest (three_phase_flash.hpp:300-489)
 * for a batch.  active[n] PhasePresence bits of the tested set,
 * compositions[3*nc*n] (same layout as nz_flash_out.composition).
 * Outputs: stable[n], valid[n], unstable_mask[n] (bit p = missing phase p
 * unstable), trial_sum[3*n], incipient[3*nc*n] (NULL to skip).
 */
int nz_stability_batch(nz_ctx* ctx, int64_t n, const double* pressure,
                       const double* temperature, const double* z,
                       const double* salinity, const uint8_t* active,
                       const double* compositions, uint8_t* stable,
                       uint8_t* valid, uint8_t* unstable_mask,
                       double* trial_sum, double* incipient, void* stream);

/* ---- Natural assembly -------------------------------------------------------
 * Cell unknowns follow Indices<FullyCompositionalThreePhase> without wells
 * (indices/include/indices/indices.hpp:30-45): B = 3*nc+1 doubles per cell
 *   [p, x_o[0..nc-2], x_g[0..nc-2], x_w[0..nc-2], S_o, S_g, S_w]
 * Phase state: 3*nc+8 doubles per cell (PetscPhaseStateCodec layout)
 *   [flag, K_g[nc], K_w[nc], z[nc], beta[3], Z[3], suppression]
 * Both are cell-major (AoS), exactly the PETSc Vec block layout.
 */
typedef struct nz_relperm_desc {
    /* Quadratic (Corey-2) curves with end points, as in the reference's
     * H2O-CO2-nC10 benchmark (case/h2o_co2_nc10_2d_benchmark/benchmark_common.hpp:97-126). */
    double swc, sorw, sgc, sorg;
    double krw_max, krg_max, kro_max;
} nz_relperm_desc;

typedef struct nz_natural_desc {
    int64_t ncell;
    const double* porosity;         /* [ncell] host */
    const double* volume;           /* [ncell] host */
    const int64_t* conn_offset;     /* [ncell+1] CSR of directed connections, host */
    const int64_t* conn_neighbor;   /* [nconn] */
    const double* conn_trans;       /* [nconn] TPFA transmissibility */
    const double* conn_gravity;     /* [nconn] g*(z_c - z_n) */
    double time_step;               /* s */
    double fugacity_scaling;        /* fugacityScalingFactor (1) */
    double temperature;             /* reservoir temperature, K */
    nz_relperm_desc relperm;
} nz_natural_desc;

typedef struct nz_natural nz_natural;

/* StateUpdateReport (natural_petsc_runtime_state.inc:280-299) */
typedef struct nz_report {
    int32_t succeeded;
    int64_t first_failure_cell;
    int32_t status;                  /* PhaseUpdateStatus of the first failure */
    int32_t phase_removed;
    int32_t missing_phase_unstable;
    int32_t stability_invalid;
    int32_t restricted_flash_failed;
    int32_t unrestricted_flash_failed;
    int64_t updated_cells;
    int64_t stable_reduced_cells;
    int64_t failed_cells;
} nz_report;

int nz_natural_create(nz_ctx* ctx, const nz_natural_desc* desc, nz_natural** out);
int nz_natural_destroy(nz_natural* nat);
/* Block-CSR pattern of the Jacobian: row_ptr[ncell+1], col_idx[nnzb]
 * (columns sorted, self included).  nnzb via *nnzb when col_idx is NULL. */
int nz_natural_pattern(nz_natural* nat, int64_t* row_ptr, int64_t* col_idx,
                       int64_t* nnzb);
/* Per-cell P-T-z initialisation: flashPTZ + assignFlashResult into a default
 * phase state, as NaturalPetscRuntime::initializeUniformFromPTZ
 * (natural_petsc_runtime_state.inc:107-164) does for one uniform (P, z), here
 * with one (P, z) per cell.  P[ncell], z[ncell][nc] (cell-major), primary and
 * phase_state outputs, all device pointers.  Returns NZ_RECOVERABLE, with
 * *first_failure = the lowest failing cell, when a flash does not converge
 * (the reference throws); nothing is written then.  Unless the per-cell
 * update mode is set (nz_natural_set_update_mode), every cell's flash runs
 * through the batched staged flash first, in a work space allocated for the
 * call (about 2.5 KB per cell for nc = 3). */
int nz_natural_init_ptz(nz_natural* nat, const double* P, const double* z,
                        double* primary, double* phase_state,
                        int64_t* first_failure, void* stream);
/* Accepted history: previous-time accumulation M^n from primary/phase state
 * (refreshPreviousPropertiesCache_, natural_petsc_runtime_cache_history.inc:180-262). */
int nz_natural_set_history(nz_natural* nat, const double* primary,
                           const double* phase_state, void* stream);
/* Transactional phase-state update of every cell; commits all cells or none.
 * Two equivalent forms (same results):
 *   staged    every cell's stability test runs on the batched lane-per-trial
 *             kernels and every reflash on the staged batched flash, then the
 *             per-cell code takes those answers (work space held by the
 *             nz_natural from its creation: about 2.8 KB per cell for nc = 3,
 *             5.0 KB for nc = 6, 6.8 KB for nc = 8, plus the reflash batch's,
 *             grown on demand; one host synchronisation to size that batch);
 *   per-cell  each cell runs its whole update in one thread (a warp per cell
 *             on grids below 256 cells per SM).
 * NZ_UPDATE_AUTO (the default) takes the staged form from 256 cells per SM,
 * where the per-cell form runs one thread per cell. */
int nz_update_state(nz_natural* nat, double* primary, double* phase_state,
                    nz_report* report, void* stream);
#define NZ_UPDATE_PER_CELL 0
#define NZ_UPDATE_STAGED 1
#define NZ_UPDATE_AUTO 2
int nz_natural_set_update_mode(nz_natural* nat, int32_t mode);
/* Residual F[ncell*B] (cell-major). */
int nz_residual(nz_natural* nat, const double* primary,
                const double* phase_state, double* residual, void* stream);
/* BAIJ values in pattern order, each block B*B row-major (the layout
 * MatSetValuesBlocked takes); residual may be NULL. */
int nz_jacobian(nz_natural* nat, const double* primary,
                const double* phase_state, double* baij_values,
                double* residual, void* stream);
/* The same values in cell-column order, for the reference's batched block
 * write (insertPreparedCellJacobianColumn_, natural_petsc_runtime_jacobian.inc:
 * 279-299): cell c's column is the contiguous run of 1 + nconn(c) blocks that
 * starts at block c + conn_offset[c] -- the self block, then the block of each
 * of its connections in connection order -- i.e. exactly the values of
 *   MatSetValuesBlocked(J, 1 + nconn(c), rows, 1, &c, vals, ADD_VALUES)
 * with rows = {c, conn_neighbor[conn_offset[c] .. conn_offset[c+1])}.
 * column_values holds nnzb * B * B doubles; residual may be NULL. */
int nz_jacobian_columns(nz_natural* nat, const double* primary,
                        const double* phase_state, double* column_values,
                        double* residual, void* stream);

/* ---- diagnostics -------------------------------------------------------------
 * Measured FMA throughput of the FP64 and FP32 CUDA-core pipes of `device`
 * (TFLOP/s, 2 flops per FMA): the roofline denominators of the flash, which
 * is bound by those pipes.  No counterpart in the reference (no GPU code).
 */
int nz_diag_fma_peak(int32_t device, double* fp64_tflops, double* fp32_tflops);

#ifdef __cplusplus
}
#endif

#endif /* NONENONE_B200_H */
