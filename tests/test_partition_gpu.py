"""The partitioned Natural assembly on the GPU, ranks emulated on one GPU.

Each rank's local domain runs on its own NaturalAssembler; the halo exchange is
done in two phases (every rank posts its sends, then every rank takes its halo)
through an in-process mailbox instead of NCCL, since only one GPU is present.
The owned rows must equal the single-domain GPU results bit for bit and the
reference's golden values within the tolerances of test_natural_gpu.py; the
combined update report must equal the single-domain report.
"""
import types

import numpy as np
import pytest

from nonenone_b200 import abi, synth
from nonenone_b200.fluids import make_fluid
from nonenone_b200.partition import (AssemblerLocal, DistributedNatural, combine_reports, post_halo,
                                     take_halo)
from tests.test_natural_gpu import assert_entries, assert_state

pytestmark = pytest.mark.gpu

REPORT_FIELDS = [f for f, _ in abi.Report._fields_]


class _Mailbox:
    def __init__(self, box, rank):
        self.box, self.rank = box, rank

    def send(self, peer, rows):
        self.box[(self.rank, peer)] = rows.clone()

    def recv(self, peer, like, n):
        out = self.box.pop((peer, self.rank))
        assert out.shape[0] == n
        return out

    def flush(self):
        pass


def _grid(g):
    return types.SimpleNamespace(
        ncell=g["porosity"].shape[0], porosity=g["porosity"], volume=g["volume"],
        conn_offset=g["conn_offset"], conn_neighbor=g["conn_neighbor"],
        conn_trans=g["conn_trans"], conn_gravity=g["conn_gravity"])


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_assembly_on_one_gpu(golden, world):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    from nonenone_b200.flash import Context
    from nonenone_b200.natural import NaturalAssembler
    g = golden("natural_pr_nc3.npz")
    grid = _grid(g)
    fluid = make_fluid()
    ctx = Context(fluid)
    relperm = abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10)
    dt, T = float(g["time_step"]), float(g["temperature"])
    dev = torch.device("cuda", 0)
    box = {}
    ranks = [DistributedNatural(grid, world, r, lambda gr: AssemblerLocal(ctx, gr, dt, T, relperm, "staged"),
                                _Mailbox(box, r)) for r in range(world)]

    def localize(P, S):
        locs = []
        for dn in ranks:
            own, nl = dn.dom.owned, dn.dom.grid.ncell
            locs.append(list(dn.place(torch.as_tensor(P[own], device=dev), torch.as_tensor(S[own], device=dev),
                                      torch.zeros(nl, P.shape[1], dtype=torch.float64, device=dev),
                                      torch.zeros(nl, S.shape[1], dtype=torch.float64, device=dev))))
        for field in (0, 1):   # two-phase exchange: all sends, then all receives
            for dn, loc in zip(ranks, locs):
                post_halo(dn.dom, loc[field], dn.comm.send)
            for dn, loc in zip(ranks, locs):
                take_halo(dn.dom, loc[field], lambda peer, n, dn=dn, x=loc[field]: dn.comm.recv(peer, x, n))
        return locs

    for dn, (p, s) in zip(ranks, localize(g["primary"], g["phase_state"])):
        dn.set_history(p, s)
    cur = localize(g["current"], g["phase_state"])
    F = torch.cat([dn.residual(p, s) for dn, (p, s) in zip(ranks, cur)]).cpu().numpy()
    J = torch.cat([dn.jacobian(p, s) for dn, (p, s) in zip(ranks, cur)]).cpu().numpy()

    # the single-domain GPU run
    whole = NaturalAssembler(ctx, grid, dt, T, relperm)
    whole.set_update_mode("staged")
    whole.refresh_history(g["primary"], g["phase_state"])
    dcur = torch.as_tensor(g["current"], device=dev)
    dps = torch.as_tensor(g["phase_state"], device=dev)
    assert np.array_equal(F, whole.form_function(dcur, dps).cpu().numpy())
    assert np.array_equal(J, whole.assemble_jacobian(dcur, dps).cpu().numpy())
    # against the reference, with the tolerances of test_natural_gpu.py
    assert_entries(F, g["residual"], 1, "partitioned residual")
    assert_entries(J, g["jacobian"], 1, "partitioned jacobian")

    for it, want in (("current", g["report"]), ("failing", g["failing_report"])):
        outs = [dn.cellwise.update(torch.as_tensor(g[it][dn.dom.owned], device=dev),
                                   torch.as_tensor(g["phase_state"][dn.dom.owned], device=dev)) for dn in ranks]
        rep = combine_reports(ranks[0].dom, [o[3] for o in outs])
        got = np.array([getattr(rep, f) for f in REPORT_FIELDS])
        assert np.array_equal(got, want), (it, dict(zip(REPORT_FIELDS, zip(got, want))))
        if it == "current":
            up = torch.cat([o[1] for o in outs]).cpu().numpy()
            ups = torch.cat([o[2] for o in outs]).cpu().numpy()
            assert_state(up, ups, g["updated_primary"], g["updated_phase_state"], "partitioned update")
