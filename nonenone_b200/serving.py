"""Continuous-batching request loop over the Natural flash + assembly path.

A request is one flash + assembly job of one model (a reservoir grid with its
fluid):

* the first request of a model builds it on the GPU -- the per-cell P-T-z
  flash of its initial state (``initialize_from_ptz``), the accepted history,
  the residual and the BAIJ Jacobian -- and leaves the model resident;
* a repeat request is the next Newton iteration of a resident model: the
  transactional phase-state update of a perturbed iterate starts from the
  model's device-resident phase state (its K-values, phase labels and
  suppression flags are the warm start), then the residual and the Jacobian.

The loop admits requests as they arrive (their arrival times are given, e.g.
a Poisson stream) onto a fixed number of slots, each a host thread with its
own CUDA stream, so work from several requests overlaps on the device.  A
request is admitted when a slot is free and the device working set stays
within the HBM budget: resident models that no queued or running request
needs are evicted, least recently used first; a request whose model alone
exceeds the budget is rejected.  Requests of one model run in arrival order,
one at a time, so every result is the one the request would give alone.

The scheduling (admission, eviction, ordering, statistics) is plain host
logic that runs with any executor; ``NaturalExecutor`` is the GPU one.
"""
from __future__ import annotations

import dataclasses
import hashlib
import math
import threading
import time
from collections import OrderedDict, deque
from typing import Callable, Dict, List, Optional

import numpy as np


@dataclasses.dataclass
class Request:
    rid: int
    model: int        # key of the (resident) model
    arrival: float    # seconds after the start of the run
    cells: int
    nc: int
    eos: str          # "pr", "sw" or "cpa"
    repeat: bool      # a repeat Newton iteration of a resident model


@dataclasses.dataclass
class Outcome:
    rid: int
    model: int
    arrival: float
    admitted: float = math.nan
    finished: float = math.nan
    queued: bool = False
    rejected: bool = False
    result: Optional[dict] = None
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def poisson_requests(n: int, rate: float, seed: int = 5, cells=(1.0e3, 1.0e6), nc_choices=(3, 4, 5, 6, 8),
                     eos_mix=(("pr", 0.5), ("sw", 0.3), ("cpa", 0.2)), repeat_fraction: float = 0.3) -> List[Request]:
    """n requests of a Poisson stream of `rate` per second: cell counts
    log-uniform in `cells`, component count uniform over `nc_choices`, EOS by
    `eos_mix`; a `repeat_fraction` of the requests (after the first) are
    repeat iterations of an earlier model, which keep its size and fluid."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out: List[Request] = []
    models: List[Request] = []
    names = [e for e, _ in eos_mix]
    weights = np.array([w for _, w in eos_mix], dtype=np.float64)
    weights /= weights.sum()
    for rid in range(n):
        t += rng.exponential(1.0 / rate)
        if models and rng.uniform() < repeat_fraction:
            base = models[int(rng.integers(len(models)))]
            out.append(Request(rid, base.model, t, base.cells, base.nc, base.eos, True))
            continue
        c = int(round(math.exp(rng.uniform(math.log(cells[0]), math.log(cells[1])))))
        req = Request(rid, len(models), t, c, int(rng.choice(nc_choices)), str(rng.choice(names, p=weights)), False)
        models.append(req)
        out.append(req)
    return out


def model_bytes(cells: int, nc: int, faces_per_cell: int = 4) -> int:
    """Device working set of one resident model: its BAIJ values (self + one
    block per face), state vectors, property cache and staged-update work
    space (about 1 KB per cell per component)."""
    B = 3 * nc + 1
    return int(cells * ((1 + faces_per_cell) * B * B * 8 + (B + 3 * nc + 8) * 8 * 4 + 1024 * nc))


class ServingLoop:
    """Admission, eviction and slot scheduling of a request stream.

    `executor` offers ``run(request, slot) -> dict`` (the job's result
    summary), ``evict(model)`` and optionally ``model_bytes(request)``.
    """

    def __init__(self, executor, slots: int = 4, hbm_budget: float = 150.0e9, admission_grace: float = 1.0e-3,
                 clock: Callable[[], float] = time.perf_counter):
        self.executor = executor
        self.slots = int(slots)
        self.budget = float(hbm_budget)
        self.grace = admission_grace
        self.clock = clock
        size = getattr(executor, "model_bytes", None)
        self.size_of = size if size is not None else (lambda r: model_bytes(r.cells, r.nc))

    def run(self, requests: List[Request]) -> List[Outcome]:
        order = sorted(requests, key=lambda r: r.arrival)
        outcomes: Dict[int, Outcome] = {r.rid: Outcome(r.rid, r.model, r.arrival) for r in order}
        upcoming = deque(order)
        waiting: deque = deque()
        resident: "OrderedDict[int, int]" = OrderedDict()   # model -> bytes, least recently used first
        running: set = set()
        state = {"used": 0, "left": len(order)}
        cv = threading.Condition()
        start = self.clock()

        def now():
            return self.clock() - start

        def release_arrivals():
            t = now()
            while upcoming and upcoming[0].arrival <= t:
                waiting.append(upcoming.popleft())

        def try_admit():
            """First admissible waiting request (FIFO, a model's requests in
            order), with memory made for it; None if there is none."""
            skipped = set()
            for idx, r in enumerate(waiting):
                if r.model in running or r.model in skipped:
                    skipped.add(r.model)
                    continue
                need = 0 if r.model in resident else self.size_of(r)
                if need > self.budget:
                    del waiting[idx]
                    out = outcomes[r.rid]
                    out.rejected = True
                    out.finished = now()
                    state["left"] -= 1
                    return "rejected"
                if state["used"] + need > self.budget:
                    needed = {w.model for w in waiting} | running
                    for m in list(resident):
                        if state["used"] + need <= self.budget:
                            break
                        if m in needed:
                            continue
                        state["used"] -= resident.pop(m)
                        self.executor.evict(m)
                if state["used"] + need > self.budget:
                    skipped.add(r.model)
                    continue
                del waiting[idx]
                if r.model not in resident:
                    resident[r.model] = need
                    state["used"] += need
                resident.move_to_end(r.model)
                running.add(r.model)
                return r
            return None

        def worker(slot: int):
            while True:
                with cv:
                    while True:
                        if state["left"] <= 0:
                            cv.notify_all()
                            return
                        release_arrivals()
                        got = try_admit()
                        if got == "rejected":
                            cv.notify_all()
                            continue
                        if got is not None:
                            req = got
                            break
                        # sleep until the next arrival or a completion
                        timeout = 0.05
                        if upcoming:
                            timeout = min(timeout, max(0.0, upcoming[0].arrival - now()))
                        cv.wait(timeout=timeout)
                    out = outcomes[req.rid]
                    out.admitted = now()
                    out.queued = out.admitted - req.arrival > self.grace
                try:
                    out.result = self.executor.run(req, slot)
                except Exception as ex:   # a failed job is reported, the loop goes on
                    out.error = f"{type(ex).__name__}: {ex}"
                with cv:
                    out.finished = now()
                    running.discard(req.model)
                    state["left"] -= 1
                    cv.notify_all()

        threads = [threading.Thread(target=worker, args=(k,), daemon=True) for k in range(self.slots)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        return [outcomes[r.rid] for r in order]


def summarize(outcomes: List[Outcome]) -> dict:
    """p50 / p99 latency (s), throughput (requests/s over the run) and the
    rejected / queued / failed fractions."""
    done = [o for o in outcomes if not o.rejected and o.error is None and not math.isnan(o.finished)]
    lat = np.array([o.latency for o in done]) if done else np.zeros(0)
    end = max((o.finished for o in outcomes if not math.isnan(o.finished)), default=0.0)
    first = min((o.arrival for o in outcomes), default=0.0)
    n = max(len(outcomes), 1)
    return {
        "requests": len(outcomes), "completed": len(done),
        "latency_s": {"p50": float(np.percentile(lat, 50)) if lat.size else None,
                      "p99": float(np.percentile(lat, 99)) if lat.size else None,
                      "max": float(lat.max()) if lat.size else None},
        "throughput_req_per_s": len(done) / max(end - first, 1e-9),
        "rejected_fraction": sum(o.rejected for o in outcomes) / n,
        "queued_fraction": sum(o.queued for o in outcomes) / n,
        "failed_fraction": sum(o.error is not None for o in outcomes) / n,
    }


def _digest(*arrays) -> str:
    h = hashlib.sha1()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


class NaturalExecutor:
    """The GPU jobs of the loop: one NaturalAssembler per resident model, one
    CUDA stream per slot, one context per fluid and slot.

    Model m's grid is a 2-D structured grid of about `cells` cells (10 m x
    10 m x 5 m, the 60x20x1 case's properties) seeded by m; its initial state
    is the per-cell P-T-z flash of seeded inputs (P ~ U[10, 30] MPa, z ~
    Dirichlet(4, 2, 1, ...)); a repeat request r updates the resident state
    from an iterate perturbed with seed r.  `keep_arrays` keeps each job's
    residual and Jacobian on the host (for equality checks)."""

    def __init__(self, device: int = 0, slots: int = 4, keep_arrays: bool = False, temperature: float = 373.15,
                 scale: float = 0.2):
        import torch
        from . import abi, synth
        self.torch = torch
        self.abi = abi
        self.synth = synth
        self.device = device
        self.streams = [torch.cuda.Stream(device=device) for _ in range(slots)]
        self.keep = keep_arrays
        self.temperature = temperature
        self.scale = scale
        self.models: Dict[int, dict] = {}
        self.contexts: Dict[tuple, object] = {}
        self.lock = threading.Lock()
        self.relperm = abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10)

    def model_bytes(self, r: Request) -> int:
        return model_bytes(r.cells, r.nc)

    def _context(self, nc: int, eos: str, slot: int):
        # a context holds the fluid; the Natural assemblers keep their own work
        # space, so models on different streams may share one
        from .flash import Context
        from .fluids import model_fluid
        key = (nc, eos)
        with self.lock:
            ctx = self.contexts.get(key)
            if ctx is None:
                ctx = self.contexts[key] = Context(model_fluid(nc, eos), device=self.device)
        return ctx

    def evict(self, model: int) -> None:
        with self.lock:
            self.models.pop(model, None)

    def _build(self, r: Request, slot: int) -> dict:
        from .grid import MILLIDARCY, StructuredGrid
        from .natural import NaturalAssembler
        torch = self.torch
        rng = np.random.default_rng(1000 + r.model)
        ny = max(1, int(round(math.sqrt(r.cells / 3.0))))
        nx = max(1, int(math.ceil(r.cells / ny)))
        n = nx * ny
        kh = 100.0 * MILLIDARCY * np.exp(rng.standard_normal(n))
        grid = StructuredGrid(nx, ny, 1, 10.0, 10.0, 5.0, np.stack([kh, kh, kh], axis=1), rng.uniform(0.15, 0.25, n))
        P = rng.uniform(10.0e6, 30.0e6, n)
        z = rng.dirichlet([4.0, 2.0] + [1.0] * (r.nc - 2), n)
        nat = NaturalAssembler(self._context(r.nc, r.eos, slot), grid, 864.0, self.temperature, self.relperm)
        for _ in range(8):
            try:
                primary, ps = nat.initialize_from_ptz(P, z, stream=self.streams[slot])
                break
            except RuntimeError as ex:
                # the reference flash does not converge at this cell's inputs:
                # it takes its neighbour's, as a simulator's initialisation would
                bad = int(str(ex).rsplit(" ", 1)[-1])
                P[bad], z[bad] = P[(bad + 1) % n], z[(bad + 1) % n]
        else:
            raise RuntimeError(f"model {r.model}: P-T-z initialisation failed")
        nat.refresh_history(primary, ps, stream=self.streams[slot])
        return {"nat": nat, "primary": primary, "ps": ps, "ncell": n}

    def run(self, r: Request, slot: int) -> dict:
        torch = self.torch
        stream = self.streams[slot]
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            m = self.models.get(r.model)
            built = False
            if m is None:
                m = self._build(r, slot)
                built = True
                with self.lock:
                    self.models[r.model] = m
            nat = m["nat"]
            rc = None
            if r.repeat:
                cur = self.synth.perturb_natural_state(m["primary"].cpu().numpy(), m["ps"].cpu().numpy(), r.nc,
                                                       r.rid, self.scale, remove_fraction=0.02)
                p = torch.as_tensor(cur, device=m["primary"].device)
                s = m["ps"].clone()
                rc, _ = nat.update_state_with_report(p, s, stream=stream)
                if rc == 0:
                    m["primary"], m["ps"] = p, s   # the accepted iterate is the next warm start
            F = nat.form_function(m["primary"], m["ps"], stream=stream)
            J = nat.assemble_jacobian(m["primary"], m["ps"], stream=stream)
            stream.synchronize()
            out = {"cells": m["ncell"], "built": built, "update_rc": rc,
                   "labels": _digest(m["ps"][:, 0].cpu().numpy()),
                   "residual": _digest(F.cpu().numpy()), "jacobian": _digest(J.cpu().numpy())}
            if self.keep:
                out["arrays"] = (F.cpu().numpy(), J.cpu().numpy())
            return out
