"""Domain decomposition of the Natural assembly over ranks (one GPU each).

The reference distributes its Natural runtime over MPI ranks with PETSc: each
rank owns a block of cells, keeps one layer of ghost cells, and forms the
residual rows and Jacobian rows of its owned cells
(``models/include/natural/petsc/detail/natural_petsc_runtime_residual.inc``,
``..._jacobian.inc``; ghost values from ``DMGlobalToLocal``).  Here:

* ownership is a contiguous range of global cell indices per rank (for the
  x-fastest numbering of a structured grid: slabs along the slowest axis);
* each rank's local domain is its owned cells plus every neighbour of an owned
  cell (the halo), numbered in ascending global order so that the upwind tie
  break on cell index (``face_flux.hpp:65-87``) sees the same order as the
  single-domain run, and each owned cell keeps its connections in their global
  order, so the owned rows are computed with exactly the single-domain
  arithmetic;
* before the residual or the Jacobian, the owners send the primaries and
  phase states of the halo cells (one exchange step, point to point);
* the Jacobian's owned rows are complete: the self block and, for every
  neighbour, the reciprocal block that the neighbour's column pass computes
  from its own state and the owned cell's frozen values -- both available
  locally;
* the phase-state update is cell-local and runs on the owned cells; the
  transaction stays all-or-nothing over all ranks (one gather of the per-rank
  reports), and because ownership is a contiguous range the combined report
  (first failing cell, cells updated and stable-reduced before it) is the
  single-domain report.

Everything here is host logic; the per-rank compute object is the GPU
``NaturalAssembler`` (``AssemblerLocal``) or, in the CPU tests, the
reference's own loops.
"""
from __future__ import annotations

import types
from typing import Callable, Dict, List

import numpy as np

from . import abi


def contiguous_ranges(ncell: int, nranks: int) -> List[range]:
    """Owned global index range of every rank (sizes differ by at most one)."""
    base, extra = divmod(ncell, nranks)
    out, start = [], 0
    for r in range(nranks):
        size = base + (1 if r < extra else 0)
        out.append(range(start, start + size))
        start += size
    return out


def _halo_of(own: range, off, nb) -> np.ndarray:
    if not len(own):
        return np.zeros(0, np.int64)
    neigh = nb[off[own.start]:off[own.stop]]
    return np.setdiff1d(np.unique(neigh), np.arange(own.start, own.stop))


class RankDomain:
    """Owned cells, halo and the local cell/connection graph of one rank."""

    def __init__(self, grid, nranks: int, rank: int):
        self.nranks, self.rank = nranks, rank
        self.ranges = contiguous_ranges(grid.ncell, nranks)
        own = self.ranges[rank]
        off, nb = np.asarray(grid.conn_offset), np.asarray(grid.conn_neighbor)
        owned = np.arange(own.start, own.stop, dtype=np.int64)
        halo = _halo_of(own, off, nb)
        self.owned = owned
        self.halo = halo
        self.cells = np.union1d(owned, halo).astype(np.int64)     # local -> global, ascending
        local_of = {int(g): i for i, g in enumerate(self.cells)}
        self.owned_local = np.searchsorted(self.cells, owned)
        self.halo_local = np.searchsorted(self.cells, halo)
        self.owner_of_halo = np.searchsorted([r.stop for r in self.ranges], halo, side="right")
        # local graph: owned cells keep all their connections in global order,
        # halo cells only those to local cells
        offsets, neighbors, trans, gravity = [0], [], [], []
        for g in self.cells:
            for k in range(off[g], off[g + 1]):
                j = int(nb[k])
                if j in local_of:
                    neighbors.append(local_of[j])
                    trans.append(grid.conn_trans[k])
                    gravity.append(grid.conn_gravity[k])
            offsets.append(len(neighbors))
        self.grid = types.SimpleNamespace(
            ncell=len(self.cells),
            porosity=np.ascontiguousarray(np.asarray(grid.porosity)[self.cells]),
            volume=np.ascontiguousarray(np.asarray(grid.volume)[self.cells]),
            conn_offset=np.asarray(offsets, np.int64),
            conn_neighbor=np.asarray(neighbors, np.int64),
            conn_trans=np.asarray(trans, np.float64),
            conn_gravity=np.asarray(gravity, np.float64))
        # the owned cells without connections: the grid of the phase-state update
        self.update_grid = types.SimpleNamespace(
            ncell=len(owned),
            porosity=np.ascontiguousarray(np.asarray(grid.porosity)[owned]),
            volume=np.ascontiguousarray(np.asarray(grid.volume)[owned]),
            conn_offset=np.zeros(len(owned) + 1, np.int64),
            conn_neighbor=np.zeros(0, np.int64), conn_trans=np.zeros(0), conn_gravity=np.zeros(0))
        # exchange plan: local rows this rank receives from / sends to every peer
        self.recv_from: Dict[int, np.ndarray] = {}
        for s in range(nranks):
            sel = self.halo_local[self.owner_of_halo == s]
            if s != rank and sel.size:
                self.recv_from[s] = sel
        self.send_to: Dict[int, np.ndarray] = {}
        for s in range(nranks):
            if s == rank:
                continue
            other = _halo_of(self.ranges[s], off, nb)
            mine = other[(other >= own.start) & (other < own.stop)]
            if mine.size:
                self.send_to[s] = np.searchsorted(self.cells, mine)

    def owned_rows(self, row_ptr) -> np.ndarray:
        """Indices, in the local BAIJ value array, of the owned rows' blocks (in
        row order: the owned slice of the global value array)."""
        row_ptr = np.asarray(row_ptr)
        if not len(self.owned_local):
            return np.zeros(0, np.int64)
        return np.concatenate([np.arange(row_ptr[i], row_ptr[i + 1]) for i in self.owned_local])


def _index(arr, idx):
    """`idx` (numpy int64) as an index for `arr` (numpy array or torch tensor)."""
    try:
        import torch
        if isinstance(arr, torch.Tensor):
            return torch.as_tensor(idx, dtype=torch.int64, device=arr.device)
    except ImportError:
        pass
    return idx


def post_halo(dom: RankDomain, local, send: Callable) -> None:
    """Send the rows of `local` that other ranks hold as halo (`send(peer, rows)`)."""
    for s, idx in dom.send_to.items():
        send(s, local[_index(local, idx)])


def take_halo(dom: RankDomain, local, recv: Callable) -> None:
    """Fill the halo rows of `local` from their owners (`recv(peer, n)`)."""
    for s, idx in dom.recv_from.items():
        local[_index(local, idx)] = recv(s, len(idx))


def exchange_halo(dom: RankDomain, local, send: Callable, recv: Callable) -> None:
    """Fill the halo rows of `local` ([ncell_local, width], the owned rows
    current) from their owners; every send is posted before the receives."""
    post_halo(dom, local, send)
    take_halo(dom, local, recv)


def combine_reports(dom: RankDomain, reports: List[abi.Report]) -> abi.Report:
    """The single-domain report from the per-rank reports of the owned ranges
    (natural_petsc_runtime_state.inc:280-299): ranks before the first failing
    cell succeeded, so their counts are complete; the failing rank's counts
    stop at that cell."""
    out = abi.Report()
    total = sum(len(r) for r in dom.ranges)
    first = None
    for rank, rep in enumerate(reports):
        if not rep.succeeded:
            g = dom.ranges[rank].start + int(rep.first_failure_cell)
            if first is None or g < first[0]:
                first = (g, rank)
    if first is None:
        out.succeeded = 1
        out.first_failure_cell = -1
        out.updated_cells = total
        out.stable_reduced_cells = sum(int(r.stable_reduced_cells) for r in reports)
        out.failed_cells = 0
        return out
    g, fr = first
    rep = reports[fr]
    out.succeeded = 0
    out.first_failure_cell = g
    for f in ("status", "phase_removed", "missing_phase_unstable", "stability_invalid",
              "restricted_flash_failed", "unrestricted_flash_failed"):
        setattr(out, f, getattr(rep, f))
    out.updated_cells = g
    out.stable_reduced_cells = sum(int(reports[r].stable_reduced_cells) for r in range(len(reports))
                                   if dom.ranges[r].stop <= g) + int(rep.stable_reduced_cells)
    out.failed_cells = 1
    return out


class TorchComm:
    """Point-to-point halo exchange and report gathering over torch.distributed
    (NCCL between GPUs, gloo on CPU).  Arrays travel as torch tensors.

    ``exchange`` issues every send and receive of one halo exchange as a single
    ``dist.batch_isend_irecv`` call: NCCL needs the send to and the receive
    from the same peer in one group, or two ranks that exchange with each other
    can both block once a message exceeds the eager buffer.  Receive buffers
    take the dtype of the array being exchanged (float64 primaries and phase
    states, integer labels alike)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def exchange(self, dom: "RankDomain", local) -> None:
        import torch
        is_tensor = isinstance(local, torch.Tensor)
        ops, recvs, keep = [], [], []
        for peer, idx in sorted(dom.send_to.items()):
            rows = local[_index(local, idx)]
            t = rows.contiguous() if is_tensor else torch.from_numpy(np.ascontiguousarray(rows))
            keep.append(t)
            ops.append(self.dist.P2POp(self.dist.isend, t, peer, group=self.group))
        for peer, idx in sorted(dom.recv_from.items()):
            shape = (len(idx),) + tuple(local.shape[1:])
            if is_tensor:
                buf = torch.empty(shape, dtype=local.dtype, device=local.device)
            else:
                buf = torch.from_numpy(np.empty(shape, dtype=np.asarray(local).dtype))
            recvs.append((idx, buf))
            ops.append(self.dist.P2POp(self.dist.irecv, buf, peer, group=self.group))
        if ops:
            for work in self.dist.batch_isend_irecv(ops):
                work.wait()
        for idx, buf in recvs:
            local[_index(local, idx)] = buf if is_tensor else buf.numpy()

    def gather_reports(self, rep: abi.Report) -> List[abi.Report]:
        fields = [f for f, _ in abi.Report._fields_]
        mine = {f: int(getattr(rep, f)) for f in fields}
        out = [None] * self.dist.get_world_size(self.group)
        self.dist.all_gather_object(out, mine, group=self.group)
        reps = []
        for d in out:
            r = abi.Report()
            for f in fields:
                setattr(r, f, d[f])
            reps.append(r)
        return reps


class DistributedNatural:
    """One rank of the partitioned Natural evaluation.

    `make(grid)` builds the rank's compute object on a local grid; it must offer
    ``set_history(p, s)``, ``residual(p, s)``, ``jacobian(p, s)``, ``pattern()``
    and ``update(p, s) -> (rc, p_new, s_new, report)`` (arrays cell-major, the
    Vec layouts).  `comm` offers ``exchange(dom, arr)`` (``TorchComm``) or
    ``send``, ``recv`` and ``flush``, and ``gather_reports``."""

    def __init__(self, grid, nranks: int, rank: int, make: Callable, comm):
        self.dom = RankDomain(grid, nranks, rank)
        self.comm = comm
        self.local = make(self.dom.grid)
        self.cellwise = make(self.dom.update_grid)
        rp, _ = self.local.pattern()
        self.owned_blocks = self.dom.owned_rows(rp)

    def _exchange(self, arr):
        if hasattr(self.comm, "exchange"):
            self.comm.exchange(self.dom, arr)
            return
        exchange_halo(self.dom, arr, self.comm.send, lambda peer, n: self.comm.recv(peer, arr, n))
        self.comm.flush()

    def place(self, primary_owned, ps_owned, template_p, template_s):
        """Local arrays with the owned rows set (halo rows not yet filled)."""
        p, s = template_p, template_s
        p[_index(p, self.dom.owned_local)] = primary_owned
        s[_index(s, self.dom.owned_local)] = ps_owned
        return p, s

    def localize(self, primary_owned, ps_owned, template_p, template_s):
        """Local arrays with the owned rows set and the halo rows exchanged."""
        p, s = self.place(primary_owned, ps_owned, template_p, template_s)
        self._exchange(p)
        self._exchange(s)
        return p, s

    def set_history(self, p_local, s_local):
        self.local.set_history(p_local, s_local)

    def residual(self, p_local, s_local):
        """Residual rows of the owned cells."""
        F = self.local.residual(p_local, s_local)
        return F[_index(F, self.dom.owned_local)]

    def jacobian(self, p_local, s_local):
        """BAIJ blocks of the owned rows, in the global value order."""
        J = self.local.jacobian(p_local, s_local)
        return J[_index(J, self.owned_blocks)]

    def update_state(self, primary_owned, ps_owned):
        """Transactional update of the owned cells over all ranks: returns
        (rc, primary, phase_state, report) with the single-domain report; the
        states are the originals unless every rank succeeded."""
        rc, p_new, s_new, rep = self.cellwise.update(primary_owned, ps_owned)
        combined = combine_reports(self.dom, self.comm.gather_reports(rep))
        if not combined.succeeded:
            return 1, primary_owned, ps_owned, combined
        return 0, p_new, s_new, combined


class AssemblerLocal:
    """A rank's compute object on its GPU: the NaturalAssembler of the local
    grid (primaries and phase states as torch tensors on that device)."""

    def __init__(self, ctx, grid, time_step: float, temperature: float, relperm, mode: str = "auto"):
        from .natural import NaturalAssembler
        self.nat = NaturalAssembler(ctx, grid, time_step, temperature, relperm)
        self.nat.set_update_mode(mode)

    def set_history(self, p, s):
        self.nat.refresh_history(p, s)

    def residual(self, p, s):
        return self.nat.form_function(p, s)

    def jacobian(self, p, s):
        return self.nat.assemble_jacobian(p, s)

    def pattern(self):
        return self.nat.pattern()

    def update(self, p, s):
        p2, s2 = p.clone(), s.clone()
        rc, rep = self.nat.update_state_with_report(p2, s2)
        return rc, p2, s2, rep
