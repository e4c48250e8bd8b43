"""The allocation-free flash entry point (nz_flash_batch_noalloc).

It exists for callers that must not allocate device memory while they run,
such as hosts whose GPU memory is held by another allocator's pool.  Its work
space is a fixed static device array, so these tests check that it returns
what the allocating entry point (nz_flash_batch) returns on the same inputs
with the same precision (staged FP64 and mixed; three and six components),
on two calls in a row (the array keeps the previous call's contents), that
those answers meet the reference's on the committed fixtures, and that a
batch larger than the array is refused cleanly.  The
file sorts last so a run that stops at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from nonenone_b200 import abi
from nonenone_b200.fluids import SIX_COMPONENT, make_fluid

pytestmark = pytest.mark.gpu

TOL = 1e-8   # the flash tolerance of the other GPU tests


CASES = [("flash_pr_nc3.npz", dict(), abi.PRECISION_FP64_STAGED),
         ("flash_pr_nc3.npz", dict(), abi.PRECISION_MIXED),
         ("flash_pr_nc6.npz", dict(names=SIX_COMPONENT), abi.PRECISION_FP64_STAGED),
         ("flash_pr_nc6.npz", dict(names=SIX_COMPONENT), abi.PRECISION_MIXED)]


def _setup(golden, name, fluid_args):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    from nonenone_b200.flash import CubicThreePhaseFlash
    g = golden(name)
    fl = CubicThreePhaseFlash(make_fluid(**fluid_args))
    d = fl.device
    inputs = dict(P=torch.tensor(g["P"], device=d), T=torch.tensor(g["T"], device=d),
                  z=torch.tensor(g["z"], device=d))
    return torch, fl, inputs, g


def _noalloc(fl, inputs, n, out, torch, precision):
    fo = fl._out_struct(out)
    rc = fl.lib.nz_flash_batch_noalloc(
        fl.handle, n, C.c_void_p(inputs["P"].data_ptr()), C.c_void_p(inputs["T"].data_ptr()),
        C.c_void_p(inputs["z"].data_ptr()), None, C.byref(fo), precision,
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc


@pytest.mark.parametrize("name,fluid_args,precision", CASES)
def test_noalloc_matches_allocating_entry_point_twice(golden, name, fluid_args, precision):
    from tests.test_flash_gpu import compare_flash
    torch, fl, inputs, g = _setup(golden, name, fluid_args)
    n = g["P"].shape[0]
    want = fl.flash(inputs["P"], inputs["T"], inputs["z"], precision=precision)
    want = {k: v.cpu().numpy() for k, v in want.items()}
    for call in range(2):
        out = fl.allocate(n)
        rc = _noalloc(fl, inputs, n, out, torch, precision)
        assert rc == 0, fl.lib.nz_last_error().decode()
        got = {k: v.cpu().numpy() for k, v in out.items()}
        assert np.array_equal(got["status"], want["status"]), call
        assert np.array_equal(got["presence"], want["presence"]), call
        ok = want["status"] == 0
        for key in ("beta", "composition", "saturation"):
            err = np.abs(got[key][..., ok] - want[key][..., ok]) / np.maximum(1.0, np.abs(want[key][..., ok]))
            assert err.max() <= TOL, (call, key, err.max())
        # and against the reference's own answers on the committed fixture
        compare_flash(got, g)


def test_noalloc_refuses_batches_beyond_its_work_space(golden):
    torch, fl, inputs, g = _setup(golden, "flash_pr_nc3.npz", dict())
    big = 1 << 20
    fo = abi.FlashOut()
    rc = fl.lib.nz_flash_batch_noalloc(
        fl.handle, big, C.c_void_p(inputs["P"].data_ptr()), C.c_void_p(inputs["T"].data_ptr()),
        C.c_void_p(inputs["z"].data_ptr()), None, C.byref(fo), abi.PRECISION_FP64_STAGED, None)
    assert rc == abi.NZ_ERR_ARGUMENT
    msg = fl.lib.nz_last_error()
    assert b"work space" in msg
    # the limit the header documents for nc = 3 with a water component
    assert b"at most 13980 points for nc=3" in msg, msg
