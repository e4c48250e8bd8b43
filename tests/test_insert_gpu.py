"""The C ABI used from C++ the way the reference's PETSc runtime would use it.

tests/c/natural_insert.cpp is a plain C++ host program, compiled here against
include/nonenone_b200.h and the in-tree library.  It assembles the Natural
Jacobian of a committed fixture grid and inserts it into a block-CSR matrix
twice -- one batched column write per cell (MatSetValuesBlocked(J, 1+nnbr,
rows, 1, &col, vals, ADD_VALUES), the reference's
insertPreparedCellJacobianColumn_, natural_petsc_runtime_jacobian.inc:279-299)
from nz_jacobian_columns, and one block at a time from nz_jacobian -- and
compares both with the reference's captured matrix (1e-9 relative, with the
per-equation-row floor of the other Natural tests).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "natural_insert.cpp")
PKG = os.path.join(ROOT, "nonenone_b200")


def _build(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = str(tmp_path / "natural_insert")
    cmd = [cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
           SRC, "-o", exe, "-L", PKG, "-lnonenone_b200", f"-Wl,-rpath,{PKG}",
           "-L", os.path.join(cuda, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.join(cuda, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def _write_case(d, fixture, fluid, relperm):
    g = np.load(os.path.join(ROOT, "tests", "golden", fixture))
    os.makedirs(d, exist_ok=True)
    open(os.path.join(d, "fluid.bin"), "wb").write(bytes(fluid))
    meta = np.array([float(g["time_step"]), float(g["temperature"]), 1.0,
                     relperm.swc, relperm.sorw, relperm.sgc, relperm.sorg,
                     relperm.krw_max, relperm.krg_max, relperm.kro_max], dtype=np.float64)
    meta.tofile(os.path.join(d, "meta.bin"))
    for name, key, dt in (("porosity", "porosity", np.float64), ("volume", "volume", np.float64),
                          ("conn_offset", "conn_offset", np.int64), ("conn_neighbor", "conn_neighbor", np.int64),
                          ("conn_trans", "conn_trans", np.float64), ("conn_gravity", "conn_gravity", np.float64),
                          ("primary", "primary", np.float64), ("phase_state", "phase_state", np.float64),
                          ("current", "current", np.float64), ("jacobian", "jacobian", np.float64)):
        np.ascontiguousarray(g[key], dtype=dt).tofile(os.path.join(d, name + ".bin"))


def test_insert_program_builds(tmp_path):
    """The host program compiles and links against the C ABI (no GPU needed)."""
    if not os.path.exists(os.path.join(PKG, "libnonenone_b200.so")):
        pytest.skip("library not built")
    _build(tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("fixture,fluid_args", [
    ("natural_pr_nc3.npz", dict()),
    ("natural_pr_nc6.npz", dict(six=True)),
    ("natural_cpa_nc6.npz", dict(cpa6=True)),
])
def test_cpp_host_inserts_the_jacobian_like_petsc(tmp_path, fixture, fluid_args):
    from nonenone_b200 import abi, synth
    from nonenone_b200.fluids import SIX_COMPONENT, make_cpa_six, make_fluid
    exe = _build(tmp_path)
    if fluid_args.get("cpa6"):
        fluid = make_cpa_six()
    else:
        fluid = make_fluid(SIX_COMPONENT) if fluid_args.get("six") else make_fluid()
    relperm = abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10)
    case = str(tmp_path / "case")
    _write_case(case, fixture, fluid, relperm)
    r = subprocess.run([exe, case], capture_output=True, text=True, timeout=300)
    print(r.stdout.strip())
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
