"""The device flash headers built as plain C++ on the host (tests/c/host_flash.cpp).

The same source the GPU kernels run, compiled by g++, must reproduce the
reference's golden answers bit for bit on the host (status, phase labels and
phase fractions), where no FMA contraction or device libm rounding intervenes.
And the SW allocation search precomputed seed by seed into an AllocMemo (the
staged kernels' lane form) must give every point exactly the answer of the
search run in place, with the memo demonstrably read by the points that reach
the search; likewise the role-permutation search run ahead into a PermMemo.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from nonenone_b200 import abi
from nonenone_b200.fluids import SIX_COMPONENT, make_fluid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def host_flash(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("hostbuild") / "host_flash")
    subprocess.run([cxx, "-O2", "-std=c++17", "-x", "c++", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "nonenone_b200", "csrc"),
                    os.path.join(ROOT, "tests", "c", "host_flash.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    return exe


def _write_case(d, fluid, g, n=None):
    os.makedirs(d, exist_ok=True)
    opts = abi.default_flash_options()
    with open(os.path.join(d, "fluid.bin"), "wb") as fh:
        fh.write(bytes(fluid))
    with open(os.path.join(d, "opts.bin"), "wb") as fh:
        fh.write(bytes(opts))
    m = g["P"].shape[0] if n is None else n
    np.ascontiguousarray(g["P"][:m], dtype=np.float64).tofile(os.path.join(d, "P.bin"))
    np.ascontiguousarray(g["T"][:m], dtype=np.float64).tofile(os.path.join(d, "T.bin"))
    np.ascontiguousarray(g["z"][:, :m], dtype=np.float64).tofile(os.path.join(d, "z.bin"))
    if "salinity" in g:
        np.ascontiguousarray(g["salinity"][:m], dtype=np.float64).tofile(os.path.join(d, "sal.bin"))
    return m


CASES = [
    ("flash_pr_nc3.npz", lambda: make_fluid()),
    ("flash_sw_nc3.npz", lambda: make_fluid(eos_model=abi.EOS_SW)),
    ("flash_pr_nc6.npz", lambda: make_fluid(SIX_COMPONENT)),
    ("flash_continuation_pr_nc3.npz", lambda: make_fluid()),
    ("flash_boundary_sw_nc3.npz", lambda: make_fluid(eos_model=abi.EOS_SW)),
]


@pytest.mark.parametrize("name,fluid", CASES, ids=[c[0] for c in CASES])
def test_host_build_matches_reference_bit_for_bit(host_flash, tmp_path, name, fluid):
    g = dict(np.load(os.path.join(GOLDEN, name)))
    d = str(tmp_path / "case")
    n = _write_case(d, fluid(), g)
    subprocess.run([host_flash, d, "plain"], check=True, capture_output=True, text=True, timeout=600)
    presence = np.fromfile(os.path.join(d, "presence.bin"), dtype=np.uint8)
    status = np.fromfile(os.path.join(d, "status.bin"), dtype=np.uint8)
    beta = np.fromfile(os.path.join(d, "beta.bin")).reshape(3, n)
    assert np.array_equal(status, g["status"][:n])
    ok = g["status"][:n] == abi.FLASH_CONVERGED
    assert np.array_equal(presence[ok], g["presence"][:n][ok])
    assert np.array_equal(beta[:, ok], g["beta"][:, :n][:, ok])


def test_allocation_memo_replays_the_search(host_flash, tmp_path):
    g = dict(np.load(os.path.join(GOLDEN, "flash_sw_nc3.npz")))
    d = str(tmp_path / "sw")
    n = _write_case(d, make_fluid(eos_model=abi.EOS_SW), g, n=400)
    out = subprocess.run([host_flash, d, "memo"], check=True, capture_output=True, text=True,
                         timeout=900).stdout.split()
    stats = dict(zip(out[0::2], (int(v) for v in out[1::2])))
    assert stats["points"] == n
    assert stats["differ"] == 0
    # the fixture's SW mixture sends a few percent of its points to the search,
    # and at least one of them on to the role-permutation search
    assert stats["memos"] >= 5, stats
    assert stats["permuted"] >= 1, stats
