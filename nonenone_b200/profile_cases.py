"""Single workloads to run under a profiler (one process, one GPU).

  python -m nonenone_b200.profile_cases flash N [--precision fp64|fp64_staged|mixed] [--eos pr|sw]
      one N-point batch of the seeded flash mixture (after a 4,096-point warm-up
      batch, so kernels of the measured batch come second)
  python -m nonenone_b200.profile_cases natural NX NY NZ [--update] [--per-cell] [--fluid pr3|cpa6]
      P-T-z initialisation of an NX x NY x NZ grid of the H2O/CO2/nC10 case,
      then two residual + Jacobian evaluations of the accepted state; with
      --update first one transactional phase-state update of a perturbed
      iterate (staged, or with every test inside the per-cell code)
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def run_flash(n: int, precision: str, eos: str = "pr") -> None:
    import torch
    from . import abi, synth
    from .flash import CubicThreePhaseFlash
    from .fluids import make_fluid
    prec = {"fp64": abi.PRECISION_FP64, "fp64_staged": abi.PRECISION_FP64_STAGED,
            "mixed": abi.PRECISION_MIXED}[precision]
    if eos == "sw":
        fl = CubicThreePhaseFlash(make_fluid(eos_model=abi.EOS_SW, salinity=1.0))
        P, T, z, sal = synth.flash_points(n, seed=2, salinity=True)
    else:
        fl = CubicThreePhaseFlash(make_fluid())
        P, T, z = synth.flash_points(n, seed=1)
        sal = None
    w = min(n, 4096)
    fl.flash(P[:w], T[:w], np.ascontiguousarray(z[:, :w]), precision=prec,
             salinity=None if sal is None else sal[:w])
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dP, dT, dz = (torch.as_tensor(x, device=fl.device) for x in (P, T, z))
    dsal = None if sal is None else torch.as_tensor(sal, device=fl.device)
    out = fl.allocate(n)
    a.record()
    fl.flash(dP, dT, dz, precision=prec, out=out, salinity=dsal)
    b.record()
    torch.cuda.synchronize()
    print(f"flash {n} points: {a.elapsed_time(b):.1f} ms, status counts "
          f"{np.bincount(out['status'].cpu().numpy(), minlength=5).tolist()}, "
          f"{fl.eos_eval_count()} EOS evaluations")


def run_natural(nx: int, ny: int, nz: int, update: bool = False, per_cell: bool = False,
                fluid_name: str = "pr3", scale: float = 1.0) -> None:
    import time

    import torch
    from . import abi, synth
    from .flash import Context, CubicThreePhaseFlash
    from .fluids import make_cpa_six, make_fluid
    from .natural import NaturalAssembler
    t_start = time.perf_counter()
    if fluid_name == "cpa6":
        grid, P, z, depth = synth.natural_case_hydrostatic(3, nx=nx, ny=ny, nz=nz)
        fluid = make_cpa_six()
        temperature = 373.15 + 0.03 * float(np.median(depth))
    else:
        grid, P, z = synth.natural_case(0, nx=nx, ny=ny, nz=nz)
        fluid = make_fluid()
        temperature = 353.15
    ctx = Context(fluid)
    nat = NaturalAssembler(ctx, grid, 864.0, temperature, abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10))
    fl = CubicThreePhaseFlash(fluid)
    st = fl.flash(P, np.full(grid.ncell, temperature), np.ascontiguousarray(z.T),
                  precision=abi.PRECISION_FP64_STAGED)["status"].cpu().numpy()
    print(f"P-T-z flash of {grid.ncell} cells ({fluid_name}): {time.perf_counter() - t_start:.1f} s, "
          f"{int((st != 0).sum())} not converged")
    bad, good = np.where(st != 0)[0], np.where(st == 0)[0]
    P[bad], z[bad] = P[good[:bad.size]], z[good[:bad.size]]
    t0 = time.perf_counter()
    primary, ps = nat.initialize_from_ptz(P, z)
    torch.cuda.synchronize()
    print(f"initialisation of {grid.ncell} cells: {time.perf_counter() - t0:.1f} s")
    nat.refresh_history(primary, ps)
    if update:
        nat.set_update_mode("per_cell" if per_cell else "staged")
        cur = torch.as_tensor(synth.perturb_natural_state(primary.cpu().numpy(), ps.cpu().numpy(), fluid.nc, 11, scale),
                              device=primary.device)
        work_s = ps.clone()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        rc, rep = nat.update_state_with_report(cur, work_s)
        b.record()
        torch.cuda.synchronize()
        print(f"update of {grid.ncell} cells: {a.elapsed_time(b):.1f} ms, committed {rc == 0}")
    vals = torch.empty(nat.nnzb, nat.B, nat.B, dtype=torch.float64, device=primary.device)
    F = torch.empty_like(primary)
    for _ in range(2):
        nat.form_function(primary, ps, out=F)
        nat.assemble_jacobian(primary, ps, values=vals)
    torch.cuda.synchronize()
    times = {"residual": [], "jacobian": []}
    for _ in range(5):
        for key, fn in (("residual", lambda: nat.form_function(primary, ps, out=F)),
                        ("jacobian", lambda: nat.assemble_jacobian(primary, ps, values=vals))):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            times[key].append(a.elapsed_time(b))
    jac_ms = sorted(times["jacobian"])[2]
    gb = (vals.numel() + F.numel()) * 8 / 1e9
    print(f"natural {nx}x{ny}x{nz}: {grid.ncell} cells, {nat.nnzb} blocks, "
          f"{vals.numel() * 8 / 1e9:.3f} GB of Jacobian values; residual {sorted(times['residual'])[2]:.3f} ms, "
          f"jacobian {jac_ms:.3f} ms = {gb / (jac_ms * 1e-3):.0f} GB/s; "
          f"checksum {float(vals.abs().sum()):.12e}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="case", required=True)
    f = sub.add_parser("flash")
    f.add_argument("n", type=int)
    f.add_argument("--precision", default="fp64_staged", choices=["fp64", "fp64_staged", "mixed"])
    f.add_argument("--eos", default="pr", choices=["pr", "sw"],
                   help="PR, or Soreide-Whitson with salinity ~ U[0,2] mol/kg")
    nat = sub.add_parser("natural")
    nat.add_argument("nx", type=int)
    nat.add_argument("ny", type=int)
    nat.add_argument("nz", type=int)
    nat.add_argument("--update", action="store_true")
    nat.add_argument("--per-cell", action="store_true")
    nat.add_argument("--fluid", default="pr3", choices=["pr3", "cpa6"],
                     help="pr3: H2O/CO2/nC10 PR; cpa6: the six-component PR-CPA fluid on the hydrostatic grid")
    nat.add_argument("--scale", type=float, default=1.0, help="perturbation scale of the updated iterate")
    a = ap.parse_args(argv)
    if a.case == "flash":
        run_flash(a.n, a.precision, a.eos)
    else:
        run_natural(a.nx, a.ny, a.nz, a.update, a.per_cell, a.fluid, a.scale)
    return 0


if __name__ == "__main__":
    sys.exit(main())
