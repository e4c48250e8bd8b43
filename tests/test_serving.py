"""The continuous-batching request loop (nonenone_b200.serving).

CPU tests drive the scheduler with a fake executor: every request finishes,
a model's requests run in arrival order and one at a time, the working set
never exceeds the HBM budget (idle models are evicted, least recently used
first), a model larger than the budget is rejected, and requests wait when the
slots are busy.  The GPU test runs a small mixed stream (PR / SW / PR-CPA,
three and six components, new and repeat requests) on three slots and checks
that every request's result equals the one it gives when its model's requests
run alone.
"""
import threading
import time

import pytest

from nonenone_b200 import serving


class FakeExecutor:
    def __init__(self, budget, seconds_per_cell=2e-6):
        self.lock = threading.Lock()
        self.resident = {}
        self.order = {}
        self.active = set()
        self.max_bytes = 0
        self.budget = budget
        self.k = seconds_per_cell
        self.overlap = 0
        self.errors = []

    def model_bytes(self, r):
        return r.cells * 1000

    def evict(self, model):
        with self.lock:
            if model in self.active:
                self.errors.append(f"evicted running model {model}")
            self.resident.pop(model, None)

    def run(self, r, slot):
        with self.lock:
            if r.model in self.active:
                self.errors.append(f"model {r.model} ran twice at once")
            self.active.add(r.model)
            self.overlap = max(self.overlap, len(self.active))
            self.resident[r.model] = r.cells * 1000
            self.max_bytes = max(self.max_bytes, sum(self.resident.values()))
            self.order.setdefault(r.model, []).append(r.rid)
        time.sleep(r.cells * self.k)
        with self.lock:
            self.active.discard(r.model)
        return {"rid": r.rid}


def test_scheduler_orders_admits_and_evicts():
    reqs = serving.poisson_requests(120, rate=400.0, seed=3, cells=(100, 5000), repeat_fraction=0.4)
    budget = 20_000 * 1000
    ex = FakeExecutor(budget)
    out = serving.ServingLoop(ex, slots=4, hbm_budget=budget).run(reqs)
    assert not ex.errors, ex.errors[:3]
    assert all(o.result is not None or o.rejected for o in out)
    assert ex.max_bytes <= budget
    assert ex.overlap > 1   # several slots busy at once
    by_model = {}
    for r in sorted(reqs, key=lambda r: r.arrival):
        by_model.setdefault(r.model, []).append(r.rid)
    for m, rids in ex.order.items():
        assert rids == [x for x in by_model[m] if x in rids], m
    stats = serving.summarize(out)
    assert stats["completed"] + round(stats["rejected_fraction"] * len(out)) == len(out)
    assert stats["latency_s"]["p99"] >= stats["latency_s"]["p50"] > 0.0
    assert stats["queued_fraction"] > 0.0


def test_scheduler_rejects_a_model_beyond_the_budget():
    reqs = [serving.Request(0, 0, 0.0, 100, 3, "pr", False),
            serving.Request(1, 1, 0.0, 10_000_000, 3, "pr", False),
            serving.Request(2, 0, 0.001, 100, 3, "pr", True)]
    ex = FakeExecutor(1e9, seconds_per_cell=0.0)
    out = serving.ServingLoop(ex, slots=2, hbm_budget=1e9).run(reqs)
    assert [o.rejected for o in out] == [False, True, False]
    assert out[0].result and out[2].result


def test_poisson_stream_shape():
    reqs = serving.poisson_requests(2000, rate=100.0, seed=1)
    gaps = [b.arrival - a.arrival for a, b in zip(reqs, reqs[1:])]
    assert abs(sum(gaps) / len(gaps) - 0.01) < 0.002
    assert 0.25 < sum(r.repeat for r in reqs) / len(reqs) < 0.35
    assert {r.nc for r in reqs} == {3, 4, 5, 6, 8}
    new = [r for r in reqs if not r.repeat]
    assert abs(sum(r.eos == "pr" for r in new) / len(new) - 0.5) < 0.05


@pytest.mark.gpu
def test_results_are_the_same_alone_and_in_the_mix():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    reqs = serving.poisson_requests(14, rate=200.0, seed=11, cells=(100, 1500), nc_choices=(3, 6),
                                    repeat_fraction=0.4)
    mixed = serving.ServingLoop(serving.NaturalExecutor(slots=3), slots=3, hbm_budget=8e9).run(reqs)
    assert all(o.error is None and not o.rejected for o in mixed), [o.error for o in mixed if o.error]
    assert len({r.eos for r in reqs}) >= 2
    by_rid = {o.rid: o.result for o in mixed}
    for m in sorted({r.model for r in reqs}):
        alone = [r for r in reqs if r.model == m]
        solo = serving.ServingLoop(serving.NaturalExecutor(slots=1), slots=1, hbm_budget=8e9).run(alone)
        for o in solo:
            for key in ("labels", "residual", "jacobian", "update_rc"):
                assert o.result[key] == by_rid[o.rid][key], (m, o.rid, key)
    print("[serving]", serving.summarize(mixed))
