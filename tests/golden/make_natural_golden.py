"""Generate the Natural-assembly golden fixtures of tests/golden/ from the reference.

Run where the reference tree is present and oracle/_ref is built
(python -m nonenone_b200.build --oracle).  Every output array comes from the
reference's own code through oracle/_ref/libnzref.so (its PETSc-free restatement
of the runtime loops, calling the reference's kernels); inputs are seeded
(nonenone_b200.synth), so the fixtures regenerate bit for bit.

  natural_pr_nc3.npz  12x6x2 grid (gravity faces), H2O/CO2/nC10, PR
  natural_sw_nc3.npz  6x4x2 grid, Soreide-Whitson, salinity 1 mol/kg
  natural_pr_nc6.npz  6x4x1 grid, six components, PR
  natural_cpa_nc3.npz 6x4x2 grid, PR-CPA H2O/CO2/nC10 (4C water, CO2 acceptor)
  natural_cpa_nc6.npz 4x3x2 grid, six components, PR-CPA (4C water, CO2 acceptor)

Each holds the grid arrays, the P-T-z initial state (primary, phase_state), the
history accumulation, a perturbed Newton iterate (``current``) with its residual,
BAIJ Jacobian values (pattern ``row_ptr``/``col_idx``) and phase-state update
(``updated_primary``/``updated_phase_state`` and the report), and an iterate
whose update fails (``failing``) with that report.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from nonenone_b200 import abi, synth  # noqa: E402
from nonenone_b200.fluids import SIX_COMPONENT, make_cpa_h2o_co2_nc10, make_cpa_six, make_fluid  # noqa: E402
from oracle import ref  # noqa: E402

TIME_STEP = 864.0
TEMPERATURE = 353.15
REPORT_FIELDS = [f for f, _ in abi.Report._fields_]


def report_array(rep):
    return np.array([getattr(rep, f) for f in REPORT_FIELDS], dtype=np.int64)


def failing_iterate(primary, phase_state, nc, cell):
    """A copy of ``primary`` whose update fails at ``cell``: one present phase is
    pushed below the active-set boundary (so the restricted flash runs) at a
    negative pressure, which the flash rejects."""
    p = primary.copy()
    flags = np.rint(phase_state[:, 0]).astype(np.int64)
    ph = [k for k in range(3) if (flags[cell] >> k) & 1][0]
    p[cell, 0] = -1.0e6
    p[cell, 1 + 3 * (nc - 1) + ph] = 5.0e-5
    return p


def make(name, fluid, seed, shape, alpha, scale=1.0):
    grid, P, z = synth.natural_case(seed, nx=shape[0], ny=shape[1], nz=shape[2], alpha=alpha)
    relperm = abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10)
    nat = ref.Natural(fluid, grid, TIME_STEP, TEMPERATURE, relperm)
    primary, ps = nat.init_ptz(P, z)
    nat.set_history(primary, ps)
    acc = nat.accumulation()
    cur = synth.perturb_natural_state(primary, ps, fluid.nc, seed + 1, scale)
    F = nat.residual(cur, ps)
    J = nat.jacobian(cur, ps)
    rp, ci = nat.pattern()
    rc, up, ups, rep = nat.update_state(cur, ps)
    assert rc == 0, "the golden iterate must update"
    fail_cell = grid.ncell // 2
    failing = failing_iterate(primary, ps, fluid.nc, fail_cell)
    rc_f, _, _, rep_f = nat.update_state(failing, ps)
    assert rc_f == 1 and rep_f.first_failure_cell == fail_cell
    np.savez_compressed(
        os.path.join(HERE, name),
        seed=seed, shape=np.array(shape), alpha=np.array(alpha), scale=scale,
        time_step=TIME_STEP, temperature=TEMPERATURE,
        porosity=grid.porosity, volume=grid.volume, conn_offset=grid.conn_offset,
        conn_neighbor=grid.conn_neighbor, conn_trans=grid.conn_trans,
        conn_gravity=grid.conn_gravity, P=P, z=z,
        primary=primary, phase_state=ps, accumulation=acc, current=cur,
        residual=F, jacobian=J, row_ptr=rp, col_idx=ci,
        updated_primary=up, updated_phase_state=ups, report=report_array(rep),
        failing=failing, failing_report=report_array(rep_f))
    status = np.rint(ups[:, 0]).astype(int)
    print(name, "cells", grid.ncell, "blocks", rp[-1], "labels", np.bincount(status, minlength=8),
          "stable-reduced", rep.stable_reduced_cells)


def main():
    if not ref.available():
        raise SystemExit("oracle/_ref is not built")
    make("natural_pr_nc3.npz", make_fluid(), 0, (12, 6, 2), (2.0, 1.0, 1.0))
    make("natural_sw_nc3.npz", make_fluid(eos_model=abi.EOS_SW, salinity=1.0), 4, (6, 4, 2), (2.0, 1.0, 1.0))
    make("natural_pr_nc6.npz", make_fluid(SIX_COMPONENT), 5, (6, 4, 1), (4.0, 2.0, 1.0, 1.0, 1.0, 1.0))
    make("natural_cpa_nc3.npz", make_cpa_h2o_co2_nc10(), 6, (6, 4, 2), (2.0, 1.0, 1.0), scale=0.2)
    make("natural_cpa_nc6.npz", make_cpa_six(), 7, (4, 3, 2), (4.0, 2.0, 1.0, 1.0, 1.0, 1.0), scale=0.2)


if __name__ == "__main__":
    main()
