"""ctypes bindings of oracle/_ref/libnzref.so -- TEST INFRASTRUCTURE ONLY.

libnzref.so is the reference's own FP64 C++ (MPMC_SCW) compiled from its
headers by oracle/Makefile around ref_harness.cpp.  Only tests/, the smoke
check and bench.py's CPU-baseline / reference arm load it, and only as the
checker or the timed CPU baseline -- never as a product path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from nonenone_b200.abi import (FlashOut, NaturalDesc, Report, block_size,
                               default_flash_options, phase_state_size)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libnzref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"reference oracle not built: {LIB_PATH}")
        L = C.CDLL(LIB_PATH)
        vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
        L.nzref_last_error.restype = C.c_char_p
        L.nzref_flash_batch.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp, i32]
        L.nzref_eos_phase_batch.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, vp]
        L.nzref_stability_batch.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp, vp,
                                            vp, vp, vp, vp, vp, i32]
        L.nzref_boundary_distance.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp, vp, vp, i32]
        L.nzref_natural_create.argtypes = [vp, vp]
        L.nzref_natural_create.restype = vp
        L.nzref_natural_destroy.argtypes = [vp]
        for name in ("nzref_natural_init_ptz",):
            getattr(L, name).argtypes = [vp, vp, vp, vp, vp]
        L.nzref_natural_set_history.argtypes = [vp, vp, vp]
        L.nzref_natural_accumulation.argtypes = [vp, vp]
        L.nzref_update_state.argtypes = [vp, vp, vp, vp]
        L.nzref_residual.argtypes = [vp, vp, vp, vp]
        L.nzref_jacobian.argtypes = [vp, vp, vp, vp]
        L.nzref_natural_pattern.argtypes = [vp, vp, vp, vp]
        L.nzref_natural_set_threads.argtypes = [vp, i32]
        L.nzref_natural_set_threads.restype = None
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc):
    if rc < 0:
        raise RuntimeError(f"oracle error {rc}: {lib().nzref_last_error().decode()}")
    return rc


def flash_batch(fluid, P, T, z, salinity=None, options=None, threads=1):
    """Reference CubicThreePhaseFlash::flash over a batch.

    z is (nc, n) component-major.  Returns a dict of numpy arrays in the
    nz_flash_out layout.
    """
    nc = fluid.nc
    P = np.ascontiguousarray(P, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    z = np.ascontiguousarray(z, dtype=np.float64).reshape(nc, -1)
    n = P.shape[0]
    sal = None if salinity is None else np.ascontiguousarray(salinity, dtype=np.float64)
    out = dict(
        presence=np.zeros(n, np.uint8), status=np.zeros(n, np.uint8),
        beta=np.zeros((3, n)), saturation=np.zeros((3, n)),
        composition=np.zeros((3, nc, n)), compressibility=np.zeros((3, n)),
        molar_density=np.zeros((3, n)), k_gas_oil=np.zeros((nc, n)),
        k_water_oil=np.zeros((nc, n)), iterations=np.zeros(n, np.int32))
    fo = FlashOut(*[_p(out[k]) for k, _ in FlashOut._fields_])
    opts = options if options is not None else default_flash_options()
    _check(lib().nzref_flash_batch(C.byref(fluid), C.byref(opts), n, _p(P), _p(T),
                                   _p(z), _p(sal), C.byref(fo), int(threads)))
    return out


def boundary_distance(fluid, P, T, z, out, salinity=None, options=None, threads=8):
    """Distance of converged flash answers from a phase boundary in |TPD|:
    0 when a present phase has a fraction below 1e-8 (it is appearing or
    vanishing: its tangent-plane distance is zero), else the smallest
    |1 - trialSum| over the non-trivial stationary points of the reference's
    stability trials for the missing phases (inf when there is none; NaN when
    the trials throw).  Points that did not converge, and three-phase points
    without a small phase, get inf."""
    nc = fluid.nc
    P = np.ascontiguousarray(P, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    n = P.shape[0]
    z = np.ascontiguousarray(z, dtype=np.float64).reshape(nc, n)
    pres = np.ascontiguousarray(np.where(out["status"] == 0, out["presence"], 0), dtype=np.uint8)
    comps = np.ascontiguousarray(out["composition"], dtype=np.float64).reshape(3, nc, n)
    sal = None if salinity is None else np.ascontiguousarray(salinity, dtype=np.float64)
    dist = np.zeros(n)
    opts = options if options is not None else default_flash_options()
    _check(lib().nzref_boundary_distance(C.byref(fluid), C.byref(opts), n, _p(P), _p(T), _p(z), _p(sal),
                                         _p(pres), _p(comps), _p(dist), int(threads)))
    present = np.stack([(pres >> p) & 1 for p in range(3)]).astype(bool)
    small = np.any(present & (np.asarray(out["beta"]) < 1.0e-8), axis=0)
    dist[small] = 0.0
    return dist


def eos_phase_batch(fluid, P, T, x, role, salinity=None):
    nc = fluid.nc
    P = np.ascontiguousarray(P, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(nc, -1)
    role = np.ascontiguousarray(role, dtype=np.int8)
    n = P.shape[0]
    sal = None if salinity is None else np.ascontiguousarray(salinity, dtype=np.float64)
    Z = np.zeros(n)
    lnphi = np.zeros((nc, n))
    _check(lib().nzref_eos_phase_batch(C.byref(fluid), n, _p(P), _p(T), _p(x),
                                       _p(role), _p(sal), _p(Z), _p(lnphi)))
    return Z, lnphi


def stability_batch(fluid, P, T, z, active, compositions, salinity=None,
                    options=None, threads=1):
    nc = fluid.nc
    P = np.ascontiguousarray(P, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    n = P.shape[0]
    z = np.ascontiguousarray(z, dtype=np.float64).reshape(nc, n)
    active = np.ascontiguousarray(active, dtype=np.uint8)
    comps = np.ascontiguousarray(compositions, dtype=np.float64).reshape(3, nc, n)
    sal = None if salinity is None else np.ascontiguousarray(salinity, dtype=np.float64)
    r = dict(stable=np.zeros(n, np.uint8), valid=np.zeros(n, np.uint8),
             unstable_mask=np.zeros(n, np.uint8), trial_sum=np.zeros((3, n)),
             incipient=np.zeros((3, nc, n)))
    opts = options if options is not None else default_flash_options()
    _check(lib().nzref_stability_batch(
        C.byref(fluid), C.byref(opts), n, _p(P), _p(T), _p(z), _p(sal), _p(active),
        _p(comps), _p(r["stable"]), _p(r["valid"]), _p(r["unstable_mask"]),
        _p(r["trial_sum"]), _p(r["incipient"]), int(threads)))
    return r


class Natural:
    """Reference Natural runtime loops (PETSc-free) on a cell/connection graph."""

    def __init__(self, fluid, grid, time_step, temperature, relperm,
                 fugacity_scaling=1.0):
        self.fluid = fluid
        self.nc = fluid.nc
        self.B = block_size(self.nc)
        self.NPS = phase_state_size(self.nc)
        self.grid = grid
        self._keep = [grid.porosity, grid.volume, grid.conn_offset,
                      grid.conn_neighbor, grid.conn_trans, grid.conn_gravity]
        self.desc = NaturalDesc(grid.ncell, *[_p(a) for a in self._keep],
                                float(time_step), float(fugacity_scaling),
                                float(temperature), relperm)
        self.h = lib().nzref_natural_create(C.byref(fluid), C.byref(self.desc))
        if not self.h:
            raise RuntimeError(lib().nzref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().nzref_natural_destroy(self.h)
            self.h = None

    def init_ptz(self, P, z):
        n = self.grid.ncell
        primary = np.zeros((n, self.B))
        ps = np.zeros((n, self.NPS))
        P = np.ascontiguousarray(P, dtype=np.float64)
        z = np.ascontiguousarray(z, dtype=np.float64).reshape(n, self.nc)
        rc = lib().nzref_natural_init_ptz(self.h, _p(P), _p(z), _p(primary), _p(ps))
        if rc != 0:
            raise RuntimeError(f"PTz flash failed at cell {rc - 1}")
        return primary, ps

    def update_cell_seconds(self):
        """Seconds each cell's updatePhaseState took in the last update_state."""
        out = np.zeros(self.grid.ncell)
        L = lib()
        L.nzref_natural_update_cell_seconds.restype = C.c_int64
        L.nzref_natural_update_cell_seconds(self.h, _p(out))
        return out

    def set_threads(self, threads: int):
        """Worker threads of the cell loops (one kernel each); the results do
        not depend on the count."""
        lib().nzref_natural_set_threads(self.h, int(threads))

    def set_history(self, primary, ps):
        _check(lib().nzref_natural_set_history(self.h, _p(primary), _p(ps)))

    def accumulation(self):
        out = np.zeros((self.grid.ncell, self.nc))
        _check(lib().nzref_natural_accumulation(self.h, _p(out)))
        return out

    def update_state(self, primary, ps):
        primary = primary.copy()
        ps = ps.copy()
        rep = Report()
        rc = _check(lib().nzref_update_state(self.h, _p(primary), _p(ps), C.byref(rep)))
        return rc, primary, ps, rep

    def residual(self, primary, ps):
        F = np.zeros((self.grid.ncell, self.B))
        _check(lib().nzref_residual(self.h, _p(primary), _p(ps), _p(F)))
        return F

    def pattern(self):
        nnzb = C.c_int64()
        _check(lib().nzref_natural_pattern(self.h, None, None, C.byref(nnzb)))
        rp = np.zeros(self.grid.ncell + 1, np.int64)
        ci = np.zeros(nnzb.value, np.int64)
        _check(lib().nzref_natural_pattern(self.h, _p(rp), _p(ci), None))
        return rp, ci

    def jacobian(self, primary, ps):
        rp, _ = self.pattern()
        vals = np.zeros((rp[-1], self.B, self.B))
        _check(lib().nzref_jacobian(self.h, _p(primary), _p(ps), _p(vals)))
        return vals
