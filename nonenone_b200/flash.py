"""Host-side mirror of the reference's thermodynamics interface.

``CubicThreePhaseFlash`` / ``CubicEquationOfState`` keep the reference's names
and argument meaning (models/include/natural/thermo/three_phase_flash.hpp,
cubic_eos.hpp) but work on batches: every call runs one CUDA kernel through
the C ABI of include/nonenone_b200.h on torch device tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi
from .lib import check, load, require_cuda


def _ptr(t):
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())


def _dev(x, device, dtype=torch.float64):
    if x is None:
        return None
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=device)


class Context:
    """An nz_ctx: one fluid (EOS + flash options) bound to one device."""

    def __init__(self, fluid: abi.FluidDesc, options: abi.FlashOptions | None = None,
                 device: int = 0):
        require_cuda()
        self.lib = load()
        self.fluid = fluid
        self.nc = fluid.nc
        self.options = options if options is not None else abi.default_flash_options()
        self.device = torch.device("cuda", device)
        h = C.c_void_p()
        check(self.lib.nz_ctx_create(C.byref(fluid), C.byref(self.options), device, C.byref(h)),
              "nz_ctx_create")
        self.handle = h

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self.lib.nz_ctx_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stream_ptr(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class CubicEquationOfState(Context):
    def phase_result(self, pressure, temperature, x, role, salinity=None, stream=None):
        """Z[n] and ln phi[nc, n] for role 0 Oil, 1 Gas, 2 Water
        (CubicEquationOfState::phaseResult, cubic_eos.hpp:833-852)."""
        d = self.device
        P, T = _dev(pressure, d), _dev(temperature, d)
        n = P.numel()
        x = _dev(x, d).reshape(self.nc, n)
        role = _dev(role, d, torch.int8)
        sal = _dev(salinity, d)
        Z = torch.empty(n, dtype=torch.float64, device=d)
        lnphi = torch.empty(self.nc, n, dtype=torch.float64, device=d)
        check(self.lib.nz_eos_phase_batch(self.handle, n, _ptr(P), _ptr(T), _ptr(x), _ptr(role),
                                          _ptr(sal), _ptr(Z), _ptr(lnphi), _stream_ptr(stream)),
              "nz_eos_phase_batch")
        return Z, lnphi


FLASH_FIELDS = ("presence", "status", "beta", "saturation", "composition", "compressibility",
                "molar_density", "k_gas_oil", "k_water_oil", "iterations")


class CubicThreePhaseFlash(Context):
    """Batched CubicThreePhaseFlash::flash / stabilityTest on the GPU."""

    def allocate(self, n: int):
        d, nc = self.device, self.nc
        f64 = dict(dtype=torch.float64, device=d)
        return dict(
            presence=torch.empty(n, dtype=torch.uint8, device=d),
            status=torch.empty(n, dtype=torch.uint8, device=d),
            beta=torch.empty(3, n, **f64), saturation=torch.empty(3, n, **f64),
            composition=torch.empty(3, nc, n, **f64), compressibility=torch.empty(3, n, **f64),
            molar_density=torch.empty(3, n, **f64), k_gas_oil=torch.empty(nc, n, **f64),
            k_water_oil=torch.empty(nc, n, **f64),
            iterations=torch.empty(n, dtype=torch.int32, device=d))

    @staticmethod
    def _out_struct(out):
        return abi.FlashOut(*[(out[k].data_ptr() if out.get(k) is not None else None)
                              for k in FLASH_FIELDS])

    def flash(self, pressure, temperature, z, salinity=None, precision: int = abi.PRECISION_FP64,
              out=None, stream=None):
        """P [Pa] (n), T [K] (n), z (nc, n) -> dict of device tensors in the
        nz_flash_out layout (three_phase_flash.hpp:83-227)."""
        d = self.device
        P, T = _dev(pressure, d), _dev(temperature, d)
        n = P.numel()
        z = _dev(z, d).reshape(self.nc, n)
        sal = _dev(salinity, d)
        if out is None:
            out = self.allocate(n)
        fo = self._out_struct(out)
        check(self.lib.nz_flash_batch(self.handle, n, _ptr(P), _ptr(T), _ptr(z), _ptr(sal),
                                      C.byref(fo), int(precision), _stream_ptr(stream)),
              "nz_flash_batch")
        return out

    def self_check(self):
        """(queue-bound code, spin-guard code) of the last staged batch, 0 when
        none tripped; call after the batch's stream is synchronised."""
        bound, guard = C.c_int32(), C.c_int32()
        check(self.lib.nz_flash_check(self.handle, C.byref(bound), C.byref(guard)), "nz_flash_check")
        return int(bound.value), int(guard.value)

    def set_spin_limit(self, limit: int):
        """Iteration cap of the staged kernels' lane-refill loops (default 2**26)."""
        check(self.lib.nz_ctx_set_spin_limit(self.handle, int(limit)), "nz_ctx_set_spin_limit")

    def eos_eval_count(self) -> int:
        v = C.c_uint64()
        check(self.lib.nz_flash_eos_eval_count(self.handle, C.byref(v)), "nz_flash_eos_eval_count")
        return int(v.value)

    def flash_host(self, pressure, temperature, z, salinity=None, precision: int = abi.PRECISION_FP64):
        """Host numpy in/out through nz_flash_batch_host (copies inside the call)."""
        P = np.ascontiguousarray(pressure, dtype=np.float64)
        T = np.ascontiguousarray(temperature, dtype=np.float64)
        n = P.shape[0]
        z = np.ascontiguousarray(z, dtype=np.float64).reshape(self.nc, n)
        sal = None if salinity is None else np.ascontiguousarray(salinity, dtype=np.float64)
        nc = self.nc
        out = dict(presence=np.empty(n, np.uint8), status=np.empty(n, np.uint8),
                   beta=np.empty((3, n)), saturation=np.empty((3, n)),
                   composition=np.empty((3, nc, n)), compressibility=np.empty((3, n)),
                   molar_density=np.empty((3, n)), k_gas_oil=np.empty((nc, n)),
                   k_water_oil=np.empty((nc, n)), iterations=np.empty(n, np.int32))
        fo = abi.FlashOut(*[out[k].ctypes.data for k in FLASH_FIELDS])
        p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        check(self.lib.nz_flash_batch_host(self.handle, n, p(P), p(T), p(z), p(sal), C.byref(fo),
                                           int(precision)), "nz_flash_batch_host")
        return out

    def stability_test(self, pressure, temperature, z, active, compositions, salinity=None,
                       stream=None):
        """Batched stabilityTest (three_phase_flash.hpp:300-489)."""
        d, nc = self.device, self.nc
        P, T = _dev(pressure, d), _dev(temperature, d)
        n = P.numel()
        z = _dev(z, d).reshape(nc, n)
        active = _dev(active, d, torch.uint8)
        comps = _dev(compositions, d).reshape(3, nc, n)
        sal = _dev(salinity, d)
        r = dict(stable=torch.empty(n, dtype=torch.uint8, device=d),
                 valid=torch.empty(n, dtype=torch.uint8, device=d),
                 unstable_mask=torch.empty(n, dtype=torch.uint8, device=d),
                 trial_sum=torch.empty(3, n, dtype=torch.float64, device=d),
                 incipient=torch.empty(3, nc, n, dtype=torch.float64, device=d))
        check(self.lib.nz_stability_batch(
            self.handle, n, _ptr(P), _ptr(T), _ptr(z), _ptr(sal), _ptr(active), _ptr(comps),
            _ptr(r["stable"]), _ptr(r["valid"]), _ptr(r["unstable_mask"]), _ptr(r["trial_sum"]),
            _ptr(r["incipient"]), _stream_ptr(stream)), "nz_stability_batch")
        return r


def fugacity_residual(eos: "CubicEquationOfState", pressure, temperature, out, salinity=None,
                      floor: float = 1.0e-20, chunk: int = 1 << 18):
    """Largest |ln f_a - ln f_b| over the present phases of every converged
    multiphase point of a flash answer `out` (the nz_flash_out dict of device
    tensors), each phase's ln phi evaluated by the EOS entry point in its own
    role; components below `floor` in either phase are skipped.  Returns a
    float64 device tensor [n] with NaN at single-phase or failed points."""
    d = eos.device
    P = _dev(pressure, d)
    T = _dev(temperature, d)
    n = P.numel()
    sal = _dev(salinity, d)
    pres = out["presence"].to(torch.int64)
    present = torch.stack([(pres >> p) & 1 for p in range(3)]).bool()
    multi = (out["status"] == abi.FLASH_CONVERGED) & (present.sum(0) >= 2)
    res = torch.full((n,), float("nan"), dtype=torch.float64, device=d)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        m = b - a
        lnf = []
        for p in range(3):
            x = out["composition"][p][:, a:b].contiguous()
            role = torch.full((m,), p, dtype=torch.int8, device=d)
            _, lphi = eos.phase_result(P[a:b], T[a:b], x, role,
                                       salinity=None if sal is None else sal[a:b])
            lnf.append(lphi + torch.log(torch.clamp(x, min=1e-300)))
        comp = out["composition"][:, :, a:b]
        best = torch.zeros(m, dtype=torch.float64, device=d)
        for p in range(3):
            for q in range(p + 1, 3):
                both = present[p, a:b] & present[q, a:b]
                use = (comp[p] > floor) & (comp[q] > floor) & both[None, :]
                diff = torch.where(use, (lnf[p] - lnf[q]).abs(), torch.zeros_like(lnf[p]))
                best = torch.maximum(best, torch.nan_to_num(diff, nan=float("inf")).amax(0))
        res[a:b] = torch.where(multi[a:b], best, res[a:b])
    return res
