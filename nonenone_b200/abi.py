"""ctypes mirror of include/nonenone_b200.h (the C ABI of the hot path).

Only data layouts live here; loading the CUDA library is done in
``nonenone_b200.lib``.
"""
from __future__ import annotations

import ctypes as C

MAX_NC = 8

NZ_OK = 0
NZ_RECOVERABLE = 1
NZ_ERR_ARGUMENT = -1
NZ_ERR_CUDA = -2
NZ_ERR_UNSUPPORTED = -3
NZ_ERR_ALLOC = -4
NZ_ERR_SELFCHECK = -5

EOS_PR, EOS_SW, EOS_CPA = 0, 1, 2
CPA_SRK, CPA_PR = 0, 1
CPA_RADIAL_SIMPLIFIED, CPA_RADIAL_CARNAHAN_STARLING = 0, 1
SW_BIP_KIJ, SW_BIP_CONSTANT, SW_BIP_CO2, SW_BIP_HYDROCARBON, SW_BIP_CO2_CHABAB = range(5)

FLASH_CONVERGED, FLASH_FAILED, FLASH_BAD_INPUT, FLASH_EOS_ERROR, FLASH_NOT_PORTED, FLASH_UNFINISHED = range(6)

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_FP64_STAGED = 2

OIL, GAS, WATER = 0, 1, 2


class FluidDesc(C.Structure):
    _fields_ = [
        ("nc", C.c_int32),
        ("eos_model", C.c_int32),
        ("eos_type", C.c_int32),
        ("water_component", C.c_int32),
        ("omega_a", C.c_double),
        ("omega_b", C.c_double),
        ("m1", C.c_double),
        ("m2", C.c_double),
        ("minimum_composition", C.c_double),
        ("tc", C.c_double * MAX_NC),
        ("pc", C.c_double * MAX_NC),
        ("vc", C.c_double * MAX_NC),
        ("acentric", C.c_double * MAX_NC),
        ("mw", C.c_double * MAX_NC),
        ("kij", C.c_double * (MAX_NC * MAX_NC)),
        ("sw_salinity", C.c_double),
        ("sw_bip_kind", C.c_int32 * MAX_NC),
        ("sw_bip_value", C.c_double * MAX_NC),
        ("cpa_a0", C.c_double * MAX_NC),
        ("cpa_b", C.c_double * MAX_NC),
        ("cpa_c1", C.c_double * MAX_NC),
        ("cpa_epsilon", C.c_double * MAX_NC),
        ("cpa_beta", C.c_double * MAX_NC),
        ("cpa_donor_sites", C.c_int32 * MAX_NC),
        ("cpa_acceptor_sites", C.c_int32 * MAX_NC),
        ("cpa_cross_epsilon", C.c_double * (MAX_NC * MAX_NC)),
        ("cpa_cross_beta", C.c_double * (MAX_NC * MAX_NC)),
        ("cpa_physical_term", C.c_int32),
        ("cpa_radial", C.c_int32),
        ("cpa_max_association_iterations", C.c_int32),
        ("cpa_association_tolerance", C.c_double),
        ("cpa_association_damping", C.c_double),
    ]


class FlashOptions(C.Structure):
    _fields_ = [
        ("maximum_iterations", C.c_int32),
        ("maximum_rachford_rice_iterations", C.c_int32),
        ("maximum_stability_iterations", C.c_int32),
        ("stability_ssi_before_newton", C.c_int32),
        ("maximum_stability_newton", C.c_int32),
        ("two_phase_ssi_before_newton", C.c_int32),
        ("maximum_two_phase_newton", C.c_int32),
        ("three_phase_ssi_before_newton", C.c_int32),
        ("maximum_three_phase_newton", C.c_int32),
        ("fugacity_tolerance", C.c_double),
        ("rachford_rice_tolerance", C.c_double),
        ("stability_tolerance", C.c_double),
        ("phase_fraction_tolerance", C.c_double),
        ("coincident_composition_tolerance", C.c_double),
        ("composition_floor", C.c_double),
        ("log_k_step_limit", C.c_double),
        ("numerical_jacobian_step", C.c_double),
    ]


def default_flash_options() -> FlashOptions:
    """ThreePhaseFlashOptions defaults (three_phase_flash_types.hpp:21-41)."""
    return FlashOptions(120, 80, 80, 8, 12, 8, 12, 10, 12,
                        1e-9, 1e-12, 1e-9, 1e-10, 1e-8, 1e-30, 2.0, 1e-6)


class FlashOut(C.Structure):
    _fields_ = [
        ("presence", C.c_void_p),
        ("status", C.c_void_p),
        ("beta", C.c_void_p),
        ("saturation", C.c_void_p),
        ("composition", C.c_void_p),
        ("compressibility", C.c_void_p),
        ("molar_density", C.c_void_p),
        ("k_gas_oil", C.c_void_p),
        ("k_water_oil", C.c_void_p),
        ("iterations", C.c_void_p),
    ]


class ModelIO(C.Structure):
    """nz_model_io: one model's device inputs and outputs."""
    _fields_ = [
        ("pressure", C.c_void_p),
        ("temperature", C.c_void_p),
        ("z", C.c_void_p),
        ("salinity", C.c_void_p),
        ("out", FlashOut),
    ]


class RelpermDesc(C.Structure):
    _fields_ = [
        ("swc", C.c_double), ("sorw", C.c_double), ("sgc", C.c_double),
        ("sorg", C.c_double), ("krw_max", C.c_double), ("krg_max", C.c_double),
        ("kro_max", C.c_double),
    ]


class NaturalDesc(C.Structure):
    _fields_ = [
        ("ncell", C.c_int64),
        ("porosity", C.c_void_p),
        ("volume", C.c_void_p),
        ("conn_offset", C.c_void_p),
        ("conn_neighbor", C.c_void_p),
        ("conn_trans", C.c_void_p),
        ("conn_gravity", C.c_void_p),
        ("time_step", C.c_double),
        ("fugacity_scaling", C.c_double),
        ("temperature", C.c_double),
        ("relperm", RelpermDesc),
    ]


class Report(C.Structure):
    _fields_ = [
        ("succeeded", C.c_int32),
        ("first_failure_cell", C.c_int64),
        ("status", C.c_int32),
        ("phase_removed", C.c_int32),
        ("missing_phase_unstable", C.c_int32),
        ("stability_invalid", C.c_int32),
        ("restricted_flash_failed", C.c_int32),
        ("unrestricted_flash_failed", C.c_int32),
        ("updated_cells", C.c_int64),
        ("stable_reduced_cells", C.c_int64),
        ("failed_cells", C.c_int64),
    ]


def block_size(nc: int) -> int:
    """Natural unknowns per cell without wells (indices.hpp:30-45)."""
    return 3 * nc + 1


def phase_state_size(nc: int) -> int:
    """PetscPhaseStateCodec doubles per cell (indices.hpp:227-278)."""
    return 3 * nc + 8

# nz_natural_set_update_mode modes
UPDATE_PER_CELL = 0
UPDATE_STAGED = 1
UPDATE_AUTO = 2
