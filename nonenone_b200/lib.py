"""Loader of the in-tree CUDA library (libnonenone_b200.so).

There is no CPU fallback: if the library is missing, or no CUDA device is
visible, every product entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libnonenone_b200.so")

# Every symbol include/nonenone_b200.h declares.
EXPORTED = (
    "nz_flash_options_default", "nz_ctx_create", "nz_ctx_destroy", "nz_last_error",
    "nz_abi_version", "nz_eos_phase_batch", "nz_flash_batch", "nz_flash_batch_host",
    "nz_flash_eos_eval_count", "nz_stability_batch", "nz_natural_create",
    "nz_natural_destroy", "nz_natural_pattern", "nz_natural_set_history",
    "nz_update_state", "nz_residual", "nz_jacobian", "nz_diag_fma_peak",
    "nz_flash_batch_noalloc", "nz_natural_init_ptz", "nz_natural_set_update_mode",
    "nz_flash_check", "nz_ctx_set_spin_limit", "nz_jacobian_columns",
    "nz_models_create", "nz_models_destroy", "nz_models_flash", "nz_models_tune",
    "nz_models_get_tuning", "nz_models_set_tuning", "nz_models_check", "nz_models_eos_eval_count",
)

_lib = None


class NzError(RuntimeError):
    pass


def load():
    """Load (once) and return the ctypes handle; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NzError(f"CUDA library not built: {LIB_PATH} (run python -m nonenone_b200.build)")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int32
    L.nz_last_error.restype = C.c_char_p
    L.nz_abi_version.restype = i32
    L.nz_flash_options_default.argtypes = [vp]
    L.nz_flash_options_default.restype = None
    L.nz_ctx_create.argtypes = [vp, vp, i32, C.POINTER(vp)]
    L.nz_ctx_destroy.argtypes = [vp]
    L.nz_eos_phase_batch.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp]
    L.nz_flash_batch.argtypes = [vp, i64, vp, vp, vp, vp, vp, i32, vp]
    L.nz_flash_batch_host.argtypes = [vp, i64, vp, vp, vp, vp, vp, i32]
    L.nz_flash_eos_eval_count.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.nz_stability_batch.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    if hasattr(L, "nz_natural_create"):
        L.nz_natural_create.argtypes = [vp, vp, C.POINTER(vp)]
        L.nz_natural_destroy.argtypes = [vp]
        L.nz_natural_pattern.argtypes = [vp, vp, vp, vp]
        L.nz_natural_init_ptz.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.nz_natural_set_history.argtypes = [vp, vp, vp, vp]
        L.nz_update_state.argtypes = [vp, vp, vp, vp, vp]
        L.nz_natural_set_update_mode.argtypes = [vp, i32]
        L.nz_residual.argtypes = [vp, vp, vp, vp, vp]
        L.nz_jacobian.argtypes = [vp, vp, vp, vp, vp, vp]
        L.nz_jacobian_columns.argtypes = [vp, vp, vp, vp, vp, vp]
    L.nz_diag_fma_peak.argtypes = [i32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.nz_flash_batch_noalloc.argtypes = [vp, i64, vp, vp, vp, vp, vp, i32, vp]
    L.nz_flash_check.argtypes = [vp, C.POINTER(i32), C.POINTER(i32)]
    L.nz_ctx_set_spin_limit.argtypes = [vp, i64]
    L.nz_models_create.argtypes = [i32, vp, vp, vp, i32, C.POINTER(vp)]
    L.nz_models_destroy.argtypes = [vp]
    L.nz_models_flash.argtypes = [vp, vp, i32, vp]
    L.nz_models_tune.argtypes = [vp, vp, i32, i64, vp]
    L.nz_models_get_tuning.argtypes = [vp, i32, C.POINTER(i32), C.POINTER(i32)]
    L.nz_models_set_tuning.argtypes = [vp, i32, i32, i32]
    L.nz_models_check.argtypes = [vp, C.POINTER(i32), C.POINTER(i32)]
    L.nz_models_eos_eval_count.argtypes = [vp, C.POINTER(C.c_uint64)]
    if L.nz_abi_version() != 2:
        raise NzError("ABI version mismatch")
    _lib = L
    return _lib


def check(rc: int, what: str = "") -> int:
    if rc < 0:
        msg = load().nz_last_error().decode()
        raise NzError(f"{what} failed ({rc}): {msg}")
    return rc


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise NzError("no CUDA device visible: the nonenone_b200 hot path runs on the GPU only")
