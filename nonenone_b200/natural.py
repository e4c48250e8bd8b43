"""Host-side mirror of the Natural runtime's assembly loops.

``NaturalAssembler`` keeps the names and meaning of ``NaturalPetscRuntime``'s
entry points (models/include/natural/petsc/detail/natural_petsc_runtime_*.inc)
but runs every cell/face loop on the GPU through the C ABI:

* ``initialize_from_ptz``       initializeUniformFromPTZ (state.inc:107-164), per cell
* ``refresh_history``           refreshPreviousPropertiesCache_ (cache_history.inc:180-262)
* ``update_state_with_report``  updateStateWithReport (state.inc:166-345)
* ``form_function``             formFunction (residual.inc:19-133)
* ``assemble_jacobian``         assembleJacobian_ (jacobian.inc:8-299), values in the
                                block-CSR order of ``pattern()``, each block B x B row-major

Primary and phase-state arrays are cell-major device tensors ``[ncell, B]`` and
``[ncell, 3nc+8]`` (the PETSc Vec block layouts).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi
from .flash import Context, _dev, _ptr, _stream_ptr
from .lib import check

# PhaseUpdateStatus (models/include/natural/state/phase_update_result.hpp)
UPDATED, STABLE_REDUCED_SET, RECOVERABLE_THERMODYNAMIC_FAILURE = 0, 1, 2


class NaturalAssembler:
    def __init__(self, ctx: Context, grid, time_step: float, temperature: float,
                 relperm: abi.RelpermDesc, fugacity_scaling: float = 1.0):
        self.ctx = ctx
        self.lib = ctx.lib
        self.nc = ctx.nc
        self.B = abi.block_size(self.nc)
        self.NPS = 3 * self.nc + 8
        self.ncell = int(grid.ncell)
        self.device = ctx.device
        keep = [np.ascontiguousarray(a, dtype=dt) for a, dt in (
            (grid.porosity, np.float64), (grid.volume, np.float64),
            (grid.conn_offset, np.int64), (grid.conn_neighbor, np.int64),
            (grid.conn_trans, np.float64), (grid.conn_gravity, np.float64))]
        self._keep = keep
        desc = abi.NaturalDesc(self.ncell, *[a.ctypes.data_as(C.c_void_p) for a in keep],
                               float(time_step), float(fugacity_scaling), float(temperature),
                               relperm)
        h = C.c_void_p()
        check(self.lib.nz_natural_create(ctx.handle, C.byref(desc), C.byref(h)), "nz_natural_create")
        self.handle = h
        nnzb = C.c_int64()
        check(self.lib.nz_natural_pattern(h, None, None, C.byref(nnzb)), "nz_natural_pattern")
        self.nnzb = nnzb.value

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self.lib.nz_natural_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pattern(self):
        """(row_ptr[ncell+1], col_idx[nnzb]) of the block-CSR Jacobian (host int64)."""
        rp = np.zeros(self.ncell + 1, np.int64)
        ci = np.zeros(self.nnzb, np.int64)
        check(self.lib.nz_natural_pattern(self.handle, rp.ctypes.data_as(C.c_void_p),
                                          ci.ctypes.data_as(C.c_void_p), None), "nz_natural_pattern")
        return rp, ci

    def _state(self, primary, phase_state):
        p = _dev(primary, self.device).reshape(self.ncell, self.B)
        s = _dev(phase_state, self.device).reshape(self.ncell, self.NPS)
        return p, s

    def initialize_from_ptz(self, pressure, composition, stream=None):
        """Flash every cell at (P, T, z) and build its primaries and phase state.
        Returns (primary, phase_state); raises on a non-converged flash."""
        P = _dev(pressure, self.device).reshape(self.ncell)
        z = _dev(composition, self.device).reshape(self.ncell, self.nc)
        primary = torch.zeros(self.ncell, self.B, dtype=torch.float64, device=self.device)
        ps = torch.zeros(self.ncell, self.NPS, dtype=torch.float64, device=self.device)
        first = C.c_int64(-1)
        rc = check(self.lib.nz_natural_init_ptz(self.handle, _ptr(P), _ptr(z), _ptr(primary), _ptr(ps),
                                                C.byref(first), _stream_ptr(stream)),
                   "nz_natural_init_ptz")
        if rc != 0:
            raise RuntimeError(f"P-T-z flash did not converge at cell {first.value}")
        return primary, ps

    def refresh_history(self, primary, phase_state, stream=None):
        """Accept (primary, phase_state) as the previous time level."""
        p, s = self._state(primary, phase_state)
        return check(self.lib.nz_natural_set_history(self.handle, _ptr(p), _ptr(s), _stream_ptr(stream)),
                     "nz_natural_set_history")

    def set_update_mode(self, mode: str):
        """Form of update_state_with_report: "staged" (stability tests on the
        batched trial kernels, reflashes on the staged flash), "per_cell"
        (the whole update per cell) or "auto" (staged from 256 cells per SM,
        the default).  Both forms give the same results."""
        code = {"per_cell": abi.UPDATE_PER_CELL, "staged": abi.UPDATE_STAGED, "auto": abi.UPDATE_AUTO}[mode]
        check(self.lib.nz_natural_set_update_mode(self.handle, code), "nz_natural_set_update_mode")

    def update_state_with_report(self, primary, phase_state, stream=None):
        """Transactional phase-state update in place.  Returns (rc, report):
        rc 0 = committed, 1 = recoverable failure (nothing committed)."""
        rep = abi.Report()
        rc = check(self.lib.nz_update_state(self.handle, _ptr(primary), _ptr(phase_state), C.byref(rep),
                                            _stream_ptr(stream)), "nz_update_state")
        return rc, rep

    def form_function(self, primary, phase_state, out=None, stream=None):
        """Residual [ncell, B].  Raises on a domain error (a cell whose
        thermodynamics fail), which the reference reports to SNES."""
        p, s = self._state(primary, phase_state)
        F = out if out is not None else torch.empty(self.ncell, self.B, dtype=torch.float64,
                                                    device=self.device)
        rc = check(self.lib.nz_residual(self.handle, _ptr(p), _ptr(s), _ptr(F), _stream_ptr(stream)),
                   "nz_residual")
        if rc != 0:
            raise FloatingPointError("Natural residual: domain error")
        return F

    def assemble_jacobian(self, primary, phase_state, values=None, residual=None, stream=None):
        """BAIJ values [nnzb, B, B] in pattern order (and the residual when a
        tensor is passed for it)."""
        p, s = self._state(primary, phase_state)
        vals = values if values is not None else torch.empty(self.nnzb, self.B, self.B, dtype=torch.float64,
                                                             device=self.device)
        rc = check(self.lib.nz_jacobian(self.handle, _ptr(p), _ptr(s), _ptr(vals), _ptr(residual),
                                        _stream_ptr(stream)), "nz_jacobian")
        if rc != 0:
            raise FloatingPointError("Natural Jacobian: domain error")
        return vals

    def assemble_jacobian_columns(self, primary, phase_state, values=None, residual=None, stream=None):
        """The same values [nnzb, B, B] in cell-column order: cell c's self block
        and then the block of each of its connections, starting at block
        c + conn_offset[c] (the values of the reference's per-cell
        MatSetValuesBlocked column insertion, jacobian.inc:279-299)."""
        p, s = self._state(primary, phase_state)
        vals = values if values is not None else torch.empty(self.nnzb, self.B, self.B, dtype=torch.float64,
                                                             device=self.device)
        rc = check(self.lib.nz_jacobian_columns(self.handle, _ptr(p), _ptr(s), _ptr(vals), _ptr(residual),
                                                _stream_ptr(stream)), "nz_jacobian_columns")
        if rc != 0:
            raise FloatingPointError("Natural Jacobian: domain error")
        return vals
