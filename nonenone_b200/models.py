"""Uneven multi-model flash batches (the nz_models entry points).

A host that runs many independent models -- each a fluid and its cells --
calls the reference's CubicThreePhaseFlash::flash
(models/include/natural/thermo/three_phase_flash.hpp:83-227) once per cell of
each model; on the device that is one ``CubicThreePhaseFlash.flash`` per model.
``ModelBatch`` runs them together: the models of one component count share one
staged launch sequence in which every point reads its model's fluid from a
device table (PR, Soreide-Whitson and PR-CPA models mix in the same kernels),
the component-count groups run on forked streams, and the whole call is
captured once into a CUDA graph and replayed.  ``tune`` is the per-component-
count autotuner of the launch shape.  Each model's answers are those of its
own ``CubicThreePhaseFlash.flash``.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import abi
from .flash import FLASH_FIELDS, _stream_ptr
from .lib import check, load, require_cuda


class ModelBatch:
    """Models with fixed point counts: ``fluids[k]`` (an ``abi.FluidDesc``)
    with ``points[k]`` points; ``options`` None or one ``abi.FlashOptions`` per
    model."""

    def __init__(self, fluids, points, options=None, device: int = 0):
        require_cuda()
        self.lib = load()
        self.fluids = list(fluids)
        self.points = [int(n) for n in points]
        if len(self.fluids) != len(self.points) or not self.fluids:
            raise ValueError("one point count per fluid, at least one model")
        self.device = torch.device("cuda", device)
        nm = len(self.fluids)
        fl = (abi.FluidDesc * nm)(*self.fluids)
        pts = (C.c_int64 * nm)(*self.points)
        opts = None
        if options is not None:
            opts = (abi.FlashOptions * nm)(*options)
        h = C.c_void_p()
        check(self.lib.nz_models_create(nm, fl, opts, pts, device, C.byref(h)), "nz_models_create")
        self.handle = h
        self._keep = None

    def __len__(self):
        return len(self.fluids)

    def allocate(self):
        """Output dicts (the nz_flash_out layout) for every model."""
        outs = []
        for f, n in zip(self.fluids, self.points):
            d, nc = self.device, f.nc
            f64 = dict(dtype=torch.float64, device=d)
            outs.append(dict(
                presence=torch.empty(n, dtype=torch.uint8, device=d),
                status=torch.empty(n, dtype=torch.uint8, device=d),
                beta=torch.empty(3, n, **f64), saturation=torch.empty(3, n, **f64),
                composition=torch.empty(3, nc, n, **f64), compressibility=torch.empty(3, n, **f64),
                molar_density=torch.empty(3, n, **f64), k_gas_oil=torch.empty(nc, n, **f64),
                k_water_oil=torch.empty(nc, n, **f64),
                iterations=torch.empty(n, dtype=torch.int32, device=d)))
        return outs

    def _io(self, inputs, outs):
        if len(inputs) != len(self.fluids):
            raise ValueError("one input tuple per model")
        io = (abi.ModelIO * len(self.fluids))()
        keep = []
        for k, (f, n, inp) in enumerate(zip(self.fluids, self.points, inputs)):
            P, T, z = inp[0], inp[1], inp[2]
            sal = inp[3] if len(inp) > 3 else None
            for t, shape in ((P, (n,)), (T, (n,)), (z, (f.nc, n))):
                if t.device != self.device or t.dtype != torch.float64 or not t.is_contiguous() \
                        or tuple(t.shape) != shape:
                    raise ValueError(f"model {k}: inputs must be contiguous float64 {self.device} tensors "
                                     f"of shape {shape}")
            if sal is not None and (sal.device != self.device or sal.dtype != torch.float64
                                    or sal.numel() != n or not sal.is_contiguous()):
                raise ValueError(f"model {k}: salinity must be a contiguous float64 tensor of {n} points")
            io[k].pressure, io[k].temperature, io[k].z = P.data_ptr(), T.data_ptr(), z.data_ptr()
            io[k].salinity = None if sal is None else sal.data_ptr()
            o = outs[k]
            io[k].out = abi.FlashOut(*[(o[key].data_ptr() if o.get(key) is not None else None)
                                       for key in FLASH_FIELDS])
            keep.append((P, T, z, sal, o))
        return io, keep

    def flash(self, inputs, precision: int = abi.PRECISION_FP64_STAGED, outs=None, stream=None):
        """inputs[k] = (P[n], T[n], z[nc, n][, salinity[n]]) device tensors of
        model k; returns (and fills) one output dict per model.  Stream
        ordered: the inputs must stay alive until the stream reaches the call."""
        if outs is None:
            outs = self.allocate()
        io, keep = self._io(inputs, outs)
        check(self.lib.nz_models_flash(self.handle, io, precision, _stream_ptr(stream)), "nz_models_flash")
        self._keep = keep
        return outs

    def tune(self, inputs, precision: int = abi.PRECISION_FP64_STAGED, sample_points: int = 16384,
             stream=None, outs=None):
        """Per component count, time candidate launch shapes on a strided
        sample of that group's points and keep the fastest; returns
        {nc: (lane_blocks_per_sm, warp_blocks_per_sm)}."""
        if outs is None:
            outs = self.allocate()
        io, keep = self._io(inputs, outs)
        check(self.lib.nz_models_tune(self.handle, io, precision, int(sample_points), _stream_ptr(stream)),
              "nz_models_tune")
        return {nc: self.tuning(nc) for nc in sorted({f.nc for f, n in zip(self.fluids, self.points) if n > 0})}

    def tuning(self, nc: int):
        lane, warp = C.c_int32(), C.c_int32()
        check(self.lib.nz_models_get_tuning(self.handle, nc, C.byref(lane), C.byref(warp)),
              "nz_models_get_tuning")
        return lane.value, warp.value

    def set_tuning(self, nc: int, lane_blocks_per_sm: int, warp_blocks_per_sm: int):
        check(self.lib.nz_models_set_tuning(self.handle, nc, lane_blocks_per_sm, warp_blocks_per_sm),
              "nz_models_set_tuning")

    def self_check(self):
        """(queue-bound code, spin-guard code) of the last call, 0 = none tripped."""
        b, g = C.c_int32(), C.c_int32()
        self.lib.nz_models_check(self.handle, C.byref(b), C.byref(g))
        return b.value, g.value

    def eos_eval_count(self) -> int:
        v = C.c_uint64()
        check(self.lib.nz_models_eos_eval_count(self.handle, C.byref(v)), "nz_models_eos_eval_count")
        return int(v.value)

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self.lib.nz_models_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
