"""The allocation-free flash entry point (nz_flash_batch_noalloc).

It exists for callers that must not allocate device memory while they run,
such as hosts whose GPU memory is held by another allocator's pool.  Its work
space is a fixed static device array, so these tests check that it returns
what the allocating entry point (nz_flash_batch, staged FP64 form) returns on
the same inputs, on two calls in a row (the array keeps the previous call's
contents), and that a batch larger than the array is refused cleanly.  The
file sorts last so a run that stops at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from nonenone_b200 import abi
from nonenone_b200.fluids import make_fluid

pytestmark = pytest.mark.gpu

TOL = 1e-8   # the flash tolerance of the other GPU tests


@pytest.fixture(scope="module")
def setup(golden):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    from nonenone_b200.flash import CubicThreePhaseFlash
    g = golden("flash_pr_nc3.npz")
    fl = CubicThreePhaseFlash(make_fluid())
    d = fl.device
    inputs = dict(P=torch.tensor(g["P"], device=d), T=torch.tensor(g["T"], device=d),
                  z=torch.tensor(g["z"], device=d))
    return torch, fl, inputs, g["P"].shape[0]


def _noalloc(fl, inputs, n, out, torch):
    fo = fl._out_struct(out)
    rc = fl.lib.nz_flash_batch_noalloc(
        fl.handle, n, C.c_void_p(inputs["P"].data_ptr()), C.c_void_p(inputs["T"].data_ptr()),
        C.c_void_p(inputs["z"].data_ptr()), None, C.byref(fo), abi.PRECISION_FP64_STAGED,
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc


def test_noalloc_matches_allocating_entry_point_twice(setup):
    torch, fl, inputs, n = setup
    want = fl.flash(inputs["P"], inputs["T"], inputs["z"], precision=abi.PRECISION_FP64_STAGED)
    want = {k: v.cpu().numpy() for k, v in want.items()}
    for call in range(2):
        out = fl.allocate(n)
        rc = _noalloc(fl, inputs, n, out, torch)
        assert rc == 0, fl.lib.nz_last_error().decode()
        got = {k: v.cpu().numpy() for k, v in out.items()}
        assert np.array_equal(got["status"], want["status"]), call
        assert np.array_equal(got["presence"], want["presence"]), call
        ok = want["status"] == 0
        for key in ("beta", "composition", "saturation"):
            err = np.abs(got[key][..., ok] - want[key][..., ok]) / np.maximum(1.0, np.abs(want[key][..., ok]))
            assert err.max() <= TOL, (call, key, err.max())


def test_noalloc_refuses_batches_beyond_its_work_space(setup):
    torch, fl, inputs, n = setup
    big = 1 << 20
    fo = abi.FlashOut()
    rc = fl.lib.nz_flash_batch_noalloc(
        fl.handle, big, C.c_void_p(inputs["P"].data_ptr()), C.c_void_p(inputs["T"].data_ptr()),
        C.c_void_p(inputs["z"].data_ptr()), None, C.byref(fo), abi.PRECISION_FP64_STAGED, None)
    assert rc == abi.NZ_ERR_ARGUMENT
    msg = fl.lib.nz_last_error()
    assert b"work space" in msg
    # the limit the header documents for nc = 3 with a water component
    assert b"at most 14026 points for nc=3" in msg, msg
