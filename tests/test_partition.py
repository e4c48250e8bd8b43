"""Domain decomposition of the Natural assembly (nonenone_b200.partition) on CPU.

The partition logic is host code; these tests drive it with the reference's own
loops (the oracle) as the per-rank compute and torch.distributed over gloo with
2 and 3 ranks as the exchange, on the 12x6x2 golden case.  Every owned residual
row, owned Jacobian block row and owned updated state must equal the
single-domain reference result bit for bit, and the combined update report must
equal the single-domain report, for the committed iterate and for the iterate
whose update fails.
"""
import os
import socket
import types

import numpy as np
import pytest

from nonenone_b200 import abi, synth
from nonenone_b200.fluids import make_fluid
from nonenone_b200.partition import RankDomain, combine_reports, contiguous_ranges

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "natural_pr_nc3.npz")
REPORT_FIELDS = [f for f, _ in abi.Report._fields_]


def _grid(g):
    return types.SimpleNamespace(
        ncell=g["porosity"].shape[0], porosity=g["porosity"], volume=g["volume"],
        conn_offset=g["conn_offset"], conn_neighbor=g["conn_neighbor"],
        conn_trans=g["conn_trans"], conn_gravity=g["conn_gravity"])


def _load():
    with np.load(GOLDEN) as f:
        return {k: f[k] for k in f.files}


@pytest.mark.parametrize("nranks", [1, 2, 3, 5])
def test_rank_domains_cover_the_grid_and_agree_on_the_exchange(nranks):
    g = _load()
    grid = _grid(g)
    doms = [RankDomain(grid, nranks, r) for r in range(nranks)]
    owned = np.concatenate([d.owned for d in doms])
    assert np.array_equal(owned, np.arange(grid.ncell))
    for d in doms:
        assert np.intersect1d(d.owned, d.halo).size == 0
        assert np.all(np.diff(d.cells) > 0)   # ascending global order
        # every owned cell keeps all its connections, in their global order
        for lo, gcell in zip(d.owned_local, d.owned):
            a, b = grid.conn_offset[gcell], grid.conn_offset[gcell + 1]
            la, lb = d.grid.conn_offset[lo], d.grid.conn_offset[lo + 1]
            assert np.array_equal(d.cells[d.grid.conn_neighbor[la:lb]], grid.conn_neighbor[a:b])
            assert np.array_equal(d.grid.conn_trans[la:lb], grid.conn_trans[a:b])
    for r, d in enumerate(doms):
        for s, idx in d.send_to.items():
            assert np.array_equal(d.cells[idx], doms[s].cells[doms[s].recv_from[r]])
        got = np.concatenate([d.cells[i] for i in d.recv_from.values()]) if d.recv_from else np.zeros(0)
        assert np.array_equal(np.sort(got), d.halo)


def test_combined_report_is_the_single_domain_report():
    g = _load()
    grid = _grid(g)
    dom = RankDomain(grid, 3, 0)
    ranges = contiguous_ranges(grid.ncell, 3)

    def rep(succeeded, first=-1, stable=0, status=3):
        r = abi.Report()
        r.succeeded, r.first_failure_cell, r.stable_reduced_cells = succeeded, first, stable
        r.status, r.failed_cells = (status, 1) if not succeeded else (0, 0)
        r.updated_cells = first if not succeeded else 0
        return r

    ok = combine_reports(dom, [rep(1, stable=5), rep(1, stable=7), rep(1, stable=1)])
    assert ok.succeeded == 1 and ok.stable_reduced_cells == 13 and ok.updated_cells == grid.ncell
    bad = combine_reports(dom, [rep(1, stable=5), rep(0, first=10, stable=2), rep(0, first=3, stable=0)])
    assert bad.succeeded == 0
    assert bad.first_failure_cell == ranges[1].start + 10
    assert bad.updated_cells == ranges[1].start + 10
    assert bad.stable_reduced_cells == 5 + 2 and bad.failed_cells == 1


class _OracleLocal:
    """The reference's own loops on a rank's local grid (test compute object)."""

    def __init__(self, ref, fluid, grid, g):
        relperm = abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10)
        self.n = ref.Natural(fluid, grid, float(g["time_step"]), float(g["temperature"]), relperm)

    def set_history(self, p, s):
        self.n.set_history(np.ascontiguousarray(p), np.ascontiguousarray(s))

    def residual(self, p, s):
        return self.n.residual(np.ascontiguousarray(p), np.ascontiguousarray(s))

    def jacobian(self, p, s):
        return self.n.jacobian(np.ascontiguousarray(p), np.ascontiguousarray(s))

    def pattern(self):
        return self.n.pattern()

    def update(self, p, s):
        return self.n.update_state(np.ascontiguousarray(p), np.ascontiguousarray(s))


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from nonenone_b200.partition import DistributedNatural, TorchComm
    from oracle import ref
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        g = _load()
        grid = _grid(g)
        fluid = make_fluid()
        dn = DistributedNatural(grid, world, rank, lambda gr: _OracleLocal(ref, fluid, gr, g), TorchComm())
        own = dn.dom.owned
        B, NPS = g["primary"].shape[1], g["phase_state"].shape[1]
        nl = dn.dom.grid.ncell
        hp, hs = dn.localize(g["primary"][own], g["phase_state"][own], np.zeros((nl, B)), np.zeros((nl, NPS)))
        dn.set_history(hp, hs)
        cp, cs = dn.localize(g["current"][own], g["phase_state"][own], np.zeros((nl, B)), np.zeros((nl, NPS)))
        F = dn.residual(cp, cs)
        J = dn.jacobian(cp, cs)
        rc, up, ups, rep = dn.update_state(g["current"][own], g["phase_state"][own])
        frc, fp, fs, frep = dn.update_state(g["failing"][own], g["phase_state"][own])
        # an integer array (phase labels) through the same batched exchange
        lab = np.full((nl, 2), -1, np.int32)
        lab[dn.dom.owned_local, 0] = 7 * own + 3
        lab[dn.dom.owned_local, 1] = own % 5
        dn.comm.exchange(dn.dom, lab)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), owned=own, F=F, J=J, rc=rc, up=up, ups=ups,
                 lab=lab, cells=dn.dom.cells,
                 rep=np.array([getattr(rep, f) for f in REPORT_FIELDS]), frc=frc, fp=fp, fs=fs,
                 frep=np.array([getattr(frep, f) for f in REPORT_FIELDS]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_natural_equals_single_domain(world, tmp_path):
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    g = _load()
    rp = g["row_ptr"]
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        own = d["owned"]
        a, b = own[0], own[-1] + 1
        assert np.array_equal(d["F"], g["residual"][own]), r
        assert np.array_equal(d["J"], g["jacobian"][rp[a]:rp[b]]), r
        assert int(d["rc"]) == 0
        assert np.array_equal(d["up"], g["updated_primary"][own]), r
        assert np.array_equal(d["ups"], g["updated_phase_state"][own]), r
        assert np.array_equal(d["rep"], g["report"]), (r, dict(zip(REPORT_FIELDS, zip(d["rep"], g["report"]))))
        # the failing iterate: nothing committed anywhere, the single-domain report
        assert int(d["frc"]) == 1
        assert np.array_equal(d["fp"], g["failing"][own]) and np.array_equal(d["fs"], g["phase_state"][own])
        assert np.array_equal(d["frep"], g["failing_report"]), r
        # every local row, halo included, holds its owner's integer labels
        assert d["lab"].dtype == np.int32
        assert np.array_equal(d["lab"][:, 0], 7 * d["cells"] + 3), r
        assert np.array_equal(d["lab"][:, 1], d["cells"] % 5), r
