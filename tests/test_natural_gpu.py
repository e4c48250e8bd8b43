"""GPU Natural assembly parity: P-T-z initialisation, residual, BAIJ Jacobian
and the transactional phase-state update, through the C ABI, against the
reference's own FP64 code (golden fixtures, and the live oracle at full size).

Tolerances:
  * Jacobian pattern (row_ptr / col_idx) and phase labels: bit-exact;
  * residual and Jacobian entries: |gpu - ref| <= 1e-9 * max(|ref|, 1e-6 * s_e),
    with s_e the largest |ref| of that equation row over all cells (so entries
    that are rounding noise next to their row's terms are compared absolutely);
  * primaries and phase-state values: 1e-8 relative (scale max(1, |ref|)).
"""
import types

import numpy as np
import pytest

from nonenone_b200 import abi, synth
from nonenone_b200.fluids import SIX_COMPONENT, make_cpa_h2o_co2_nc10, make_cpa_six, make_fluid

pytestmark = pytest.mark.gpu

ENTRY_TOL = 1e-9
FLOOR = 1e-6
STATE_TOL = 1e-8
REPORT_FIELDS = [f for f, _ in abi.Report._fields_]

CASES = {
    "natural_pr_nc3.npz": lambda: make_fluid(),
    "natural_sw_nc3.npz": lambda: make_fluid(eos_model=abi.EOS_SW, salinity=1.0),
    "natural_pr_nc6.npz": lambda: make_fluid(SIX_COMPONENT),
    "natural_cpa_nc3.npz": lambda: make_cpa_h2o_co2_nc10(),
    "natural_cpa_nc6.npz": lambda: make_cpa_six(),
}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    return torch


def grid_of(g):
    return types.SimpleNamespace(
        ncell=g["porosity"].shape[0], porosity=g["porosity"], volume=g["volume"],
        conn_offset=g["conn_offset"], conn_neighbor=g["conn_neighbor"],
        conn_trans=g["conn_trans"], conn_gravity=g["conn_gravity"])


def assembler(fluid, grid, time_step=864.0, temperature=353.15):
    from nonenone_b200.flash import Context
    from nonenone_b200.natural import NaturalAssembler
    ctx = Context(fluid)
    nat = NaturalAssembler(ctx, grid, time_step, temperature,
                           abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10))
    nat._ctx_keep = ctx
    nat.set_update_mode("staged")   # the parity tests run the staged form on every grid size
    return nat


def assert_entries(gpu, ref, axis_eq, what):
    """Entry-wise check with the per-equation-row floor described above."""
    gpu = np.asarray(gpu)
    ref = np.asarray(ref)
    # non-finite entries (where the reference's arithmetic overflows) must match exactly
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(gpu), fin), f"{what}: non-finite pattern differs"
    inf = np.isinf(ref)
    assert np.array_equal(gpu[inf], ref[inf]), f"{what}: infinities differ"
    assert np.array_equal(np.isnan(gpu), np.isnan(ref)), f"{what}: NaN pattern differs"
    red = tuple(a for a in range(ref.ndim) if a != axis_eq)
    scale = np.max(np.where(fin, np.abs(ref), 0.0), axis=red, keepdims=True)
    denom = np.maximum(np.abs(ref), FLOOR * scale)
    with np.errstate(invalid="ignore"):
        err = np.where(fin, np.abs(gpu - ref) / np.where(denom > 0, denom, 1.0), 0.0)
    worst = np.unravel_index(np.argmax(err), err.shape)
    under = fin & (ref != 0) & (np.abs(ref) < FLOOR * scale)
    rel = np.where(fin & (ref != 0), np.abs(gpu - ref) / np.where(ref != 0, np.abs(ref), 1.0), 0.0)
    print(f"[entries] {what}: {int(fin.sum())} entries, max err {err.max():.3e}; "
          f"{int(under.sum())} nonzero entries under the row floor "
          f"(their largest plain relative error {float(rel[under].max()) if under.any() else 0.0:.3e}); "
          f"largest plain relative error above the floor {float(rel[fin & ~under].max()):.3e}")
    assert err.max() <= ENTRY_TOL, f"{what}: max err {err.max():.3e} at {worst}: {gpu[worst]} vs {ref[worst]}"
    return err.max()


def assert_state(gpu_p, gpu_s, ref_p, ref_s, what):
    assert np.array_equal(gpu_s[:, 0], ref_s[:, 0]), (
        f"{what}: phase labels differ at cells {np.where(gpu_s[:, 0] != ref_s[:, 0])[0][:10]}")
    assert np.array_equal(gpu_s[:, -1], ref_s[:, -1]), f"{what}: suppression flags differ"
    # the compressibility recorded for an absent phase is a leftover of the
    # solver's iterations that nothing reads: compare Z of present phases only
    nc = (gpu_s.shape[1] - 8) // 3
    flags = np.rint(ref_s[:, 0]).astype(np.int64)
    keep = np.ones(gpu_s.shape, dtype=bool)
    for p in range(3):
        keep[:, 4 + 3 * nc + p] = ((flags >> p) & 1).astype(bool)
    for name, a, b, m in (("primary", gpu_p, ref_p, np.ones(gpu_p.shape, dtype=bool)),
                          ("phase_state", gpu_s, ref_s, keep)):
        err = np.where(m, np.abs(a - b) / np.maximum(1.0, np.abs(b)), 0.0)
        assert err.max() <= STATE_TOL, (what, name, err.max(), np.unravel_index(err.argmax(), err.shape))


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, golden, torch_cuda):
    g = golden(request.param)
    fluid = CASES[request.param]()
    nat = assembler(fluid, grid_of(g), float(g["time_step"]), float(g["temperature"]))
    return request.param, g, nat


def test_pattern_matches_reference(case):
    _, g, nat = case
    rp, ci = nat.pattern()
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_idx"])


def test_initialize_from_ptz(case):
    name, g, nat = case
    primary, ps = nat.initialize_from_ptz(g["P"], g["z"])
    assert_state(primary.cpu().numpy(), ps.cpu().numpy(), g["primary"], g["phase_state"], name)


def test_residual_and_jacobian(case, torch_cuda):
    torch = torch_cuda
    name, g, nat = case
    nat.refresh_history(g["primary"], g["phase_state"])
    cur = torch.as_tensor(g["current"], device="cuda")
    ps = torch.as_tensor(g["phase_state"], device="cuda")
    F = nat.form_function(cur, ps).cpu().numpy()
    assert_entries(F, g["residual"], 1, f"{name} residual")
    Fj = torch.empty_like(cur)
    J = nat.assemble_jacobian(cur, ps, residual=Fj).cpu().numpy()
    assert_entries(J, g["jacobian"], 1, f"{name} jacobian")
    assert_entries(Fj.cpu().numpy(), g["residual"], 1, f"{name} residual from the Jacobian call")


def test_update_state(case, torch_cuda):
    torch = torch_cuda
    name, g, nat = case
    cur = torch.as_tensor(g["current"], device="cuda").clone()
    ps = torch.as_tensor(g["phase_state"], device="cuda").clone()
    rc, rep = nat.update_state_with_report(cur, ps)
    assert rc == 0
    got = np.array([getattr(rep, f) for f in REPORT_FIELDS])
    assert np.array_equal(got, g["report"]), dict(zip(REPORT_FIELDS, zip(got, g["report"])))
    assert_state(cur.cpu().numpy(), ps.cpu().numpy(), g["updated_primary"], g["updated_phase_state"], name)


def test_update_state_per_cell_tests(case, torch_cuda):
    """The per-cell form of the update (every stability test and reflash
    inside the per-cell code) gives the same report and states."""
    torch = torch_cuda
    name, g, nat = case
    nat.set_update_mode("per_cell")
    try:
        for it in ("current", "failing"):
            cur = torch.as_tensor(g[it], device="cuda").clone()
            ps = torch.as_tensor(g["phase_state"], device="cuda").clone()
            rc, rep = nat.update_state_with_report(cur, ps)
            want = g["report"] if it == "current" else g["failing_report"]
            got = np.array([getattr(rep, f) for f in REPORT_FIELDS])
            assert np.array_equal(got, want), (it, dict(zip(REPORT_FIELDS, zip(got, want))))
            if it == "current":
                assert rc == 0
                assert_state(cur.cpu().numpy(), ps.cpu().numpy(), g["updated_primary"],
                             g["updated_phase_state"], name + " per-cell tests")
            else:
                assert rc == 1
    finally:
        nat.set_update_mode("staged")


def test_update_state_failure_commits_nothing(case, torch_cuda):
    torch = torch_cuda
    name, g, nat = case
    cur = torch.as_tensor(g["failing"], device="cuda").clone()
    ps = torch.as_tensor(g["phase_state"], device="cuda").clone()
    before = cur.clone(), ps.clone()
    rc, rep = nat.update_state_with_report(cur, ps)
    assert rc == 1
    got = np.array([getattr(rep, f) for f in REPORT_FIELDS])
    assert np.array_equal(got, g["failing_report"]), dict(zip(REPORT_FIELDS, zip(got, g["failing_report"])))
    assert torch.equal(cur, before[0]) and torch.equal(ps, before[1])


def test_domain_error_is_recoverable(case, torch_cuda):
    torch = torch_cuda
    _, g, nat = case
    nat.refresh_history(g["primary"], g["phase_state"])
    ps = torch.as_tensor(g["phase_state"], device="cuda").clone()
    ps[3, 0] = 0.0   # an invalid phase-presence flag: the reference throws
    cur = torch.as_tensor(g["current"], device="cuda")
    with pytest.raises(FloatingPointError):
        nat.form_function(cur, ps)
    with pytest.raises(FloatingPointError):
        nat.assemble_jacobian(cur, ps)
    # the handle stays usable after the failure
    F = nat.form_function(cur, torch.as_tensor(g["phase_state"], device="cuda")).cpu().numpy()
    assert_entries(F, g["residual"], 1, "residual after a domain error")


def test_bad_topology_is_rejected(torch_cuda):
    from nonenone_b200.lib import NzError
    grid, _, _ = synth.natural_case(0, nx=4, ny=3, nz=1)
    one_way = types.SimpleNamespace(**{k: getattr(grid, k) for k in (
        "ncell", "porosity", "volume", "conn_offset", "conn_neighbor", "conn_trans", "conn_gravity")})
    one_way.conn_neighbor = grid.conn_neighbor.copy()
    one_way.conn_neighbor[0] = 5   # cell 0 -> 5 has no reverse connection
    with pytest.raises(NzError):
        assembler(make_fluid(), one_way)


def test_full_size_parity(reference, torch_cuda):
    """The 60x20x1 case (1200 cells, 2320 faces) against the live reference."""
    torch = torch_cuda
    fluid = make_fluid()
    grid, P, z = synth.natural_case(0)
    relperm = abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10)
    oracle = reference.Natural(fluid, grid, 864.0, 353.15, relperm)
    primary, ps = oracle.init_ptz(P, z)
    oracle.set_history(primary, ps)
    cur = synth.perturb_natural_state(primary, ps, 3, 11, 1.0)
    nat = assembler(fluid, grid)
    gp, gs = nat.initialize_from_ptz(P, z)
    assert_state(gp.cpu().numpy(), gs.cpu().numpy(), primary, ps, "init 60x20x1")
    nat.refresh_history(primary, ps)
    dcur = torch.as_tensor(cur, device="cuda")
    dps = torch.as_tensor(ps, device="cuda")
    assert_entries(nat.form_function(dcur, dps).cpu().numpy(), oracle.residual(cur, ps), 1, "residual 60x20x1")
    assert_entries(nat.assemble_jacobian(dcur, dps).cpu().numpy(), oracle.jacobian(cur, ps), 1,
                   "jacobian 60x20x1")
    rc, up, ups, rep = oracle.update_state(cur, ps)
    c2, s2 = dcur.clone(), dps.clone()
    grc, grep = nat.update_state_with_report(c2, s2)
    assert grc == rc
    assert [getattr(grep, f) for f in REPORT_FIELDS] == [getattr(rep, f) for f in REPORT_FIELDS]
    assert_state(c2.cpu().numpy(), s2.cpu().numpy(), up, ups, "update 60x20x1")


def test_thread_per_cell_mode_parity(reference, torch_cuda):
    """40,000 cells: enough to switch the phase-state kernels to one thread per
    cell; initialisation and the transactional update still match the reference."""
    torch = torch_cuda
    fluid = make_fluid()
    grid, P, z = synth.natural_case(5, nx=200, ny=200, nz=1)
    # the few cells whose P-T-z flash the reference cannot converge take a
    # converged cell's inputs (its initialisation would throw otherwise)
    st = reference.flash_batch(fluid, P, np.full(grid.ncell, 353.15), np.ascontiguousarray(z.T), threads=8)["status"]
    bad, good = np.where(st != 0)[0], np.where(st == 0)[0]
    P[bad], z[bad] = P[good[:bad.size]], z[good[:bad.size]]
    relperm = abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10)
    oracle = reference.Natural(fluid, grid, 864.0, 353.15, relperm)
    primary, ps = oracle.init_ptz(P, z)
    nat = assembler(fluid, grid)
    gp, gs = nat.initialize_from_ptz(P, z)
    assert_state(gp.cpu().numpy(), gs.cpu().numpy(), primary, ps, "init 200x200x1")
    oracle.set_history(primary, ps)
    cur = synth.perturb_natural_state(primary, ps, 3, 17, 1.0)
    rc, up, ups, rep = oracle.update_state(cur, ps)
    for mode in ("per_cell", "staged"):   # one thread per cell at this size, and the staged form
        nat.set_update_mode(mode)
        c2 = torch.as_tensor(cur, device="cuda")
        s2 = torch.as_tensor(ps, device="cuda")
        grc, grep = nat.update_state_with_report(c2, s2)
        assert grc == rc, mode
        assert [getattr(grep, f) for f in REPORT_FIELDS] == [getattr(rep, f) for f in REPORT_FIELDS], mode
        assert_state(c2.cpu().numpy(), s2.cpu().numpy(), up, ups, f"update 200x200x1 {mode}")
