"""Benchmark of the batched P-T-z flash on B200 (one JSON line on rank 0).

Workload: 1,048,576 independent P-T-z points, nc = 3 (H2O/CO2/nC10), PR EOS,
seeded synthetic mixture of roughly 40/40/20 % single/two/three-phase points
(nonenone_b200.synth.flash_points).  A step is one flash of the whole batch.

  value  flashes/s with inputs resident in HBM over K steps, each step a
         distinct 1M-point batch; batches run M at a time in flight on their
         own streams (device events bracket the whole region)
  e2e    the same through nz_flash_batch_host with pinned host buffers: the
         host->device inputs and device->host results are inside the region
  roofline  the flash kernel against the measured FP64 FMA peak of the box;
         algorithmic FLOPs = executed EOS evaluations x F_eos(nc),
         F_eos(nc) = 2 nc^2 + 13 nc + 50
  cpu_baseline  the reference's own FP64 flash (oracle/_ref, compiled from the
         reference tree) on a bounded sample, all host threads

natural  one Natural Newton evaluation (phase-state update + residual + BAIJ
         Jacobian) on the 60x20x1 case beside the reference's own loops on one
         core, and on a 2,000,000-cell grid with the Jacobian's HBM roofline

--impl reference times that reference CPU flash alone (rank 0; other ranks
exit).  With --gpus N under torchrun every rank flashes its own batch (weak
scaling, no collective on the data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell flash+Jacobian evals/s (mixed vs FP64 GPU, 1e-10 fug. tol); p50/p99 latency"
UNIT = "flash evals/s"
N_POINTS = 1 << 20
NC = 3
WORKLOAD = "batched P-T-z flash, 1,048,576 points per batch, nc=3 H2O/CO2/nC10, PR EOS"


def boundary_slice():
    """The batch's near-boundary slice (5 % of the points): P bisected to a
    phase-label change of the reference flash, then offset by <= 5e-6
    relative (synth.boundary_points; committed inputs, so both arms flash the
    same points)."""
    with np.load(os.path.join(ROOT, "tests", "golden", "bench_boundary_pr_nc3.npz")) as g:
        return g["P"].copy(), g["T"].copy(), np.ascontiguousarray(g["z"])


def f_eos(nc: int) -> int:
    return 2 * nc * nc + 13 * nc + 50


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi sampling of SM clock / throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.path is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_rate(fluid, P, T, z, seconds_target: float = 15.0):
    """The reference's FP64 flash on host cores over a bounded sample."""
    from oracle import ref
    threads = os.cpu_count() or 1
    # size the sample from a quick single-thread probe of the same workload
    probe = 256
    t0 = time.perf_counter()
    ref.flash_batch(fluid, P[:probe], T[:probe], z[:, :probe], threads=1)
    per_point = (time.perf_counter() - t0) / probe
    m = int(min(P.shape[0], max(threads * 64, seconds_target * threads / max(per_point, 1e-7))))
    t0 = time.perf_counter()
    ref.flash_batch(fluid, P[:m], T[:m], z[:, :m], threads=threads)
    dt = time.perf_counter() - t0
    return {"value": m / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"first {m} of the {P.shape[0]} workload points (the seeded mixture is "
                      f"shuffled, so the sample has the workload's label mix); "
                      f"{threads} threads, one CubicThreePhaseFlash each; {dt:.1f} s",
            "single_core_us_per_flash": per_point * 1e6}


def natural_measure(local: int, reps: int, hbm_peak: float | None, with_cpu: bool, with_cpa: bool = True):
    """One Natural Newton evaluation (transactional phase-state update of a
    perturbed iterate + residual + BAIJ Jacobian) on three grids:

    * the 60x20x1 H2O/CO2/nC10 case (1200 cells, 2320 faces), PR, beside the
      reference's own loops on one host core and on all host cores;
    * a 200x200x50 grid (2,000,000 cells, 5.94 M faces) of the same fluid;
    * the 200x200x50 benchmark grid with the six-component PR-CPA fluid
      (hydrostatic P, B = 19), the Jacobian's HBM roofline and the device to
      host copy of its BAIJ values (what a host PETSc insertion needs).
    Jacobian roofline: algorithmic bytes = blocks x B^2 x 8 + residual, written
    once per evaluation.
    """
    import torch
    from nonenone_b200 import abi, synth
    from nonenone_b200.flash import CubicThreePhaseFlash, Context
    from nonenone_b200.fluids import make_cpa_six, make_fluid
    from nonenone_b200.natural import NaturalAssembler
    relperm = abi.RelpermDesc(**synth.RELPERM_H2O_CO2_NC10)
    results = {}

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        a, b = events()
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    cases = [("60x20x1", "pr3", (60, 20, 1)), ("200x200x50", "pr3", (200, 200, 50))]
    if with_cpa:
        cases.append(("200x200x50_nc6_cpa", "cpa6", (200, 200, 50)))
    for label, fluid_name, shape in cases:
        t_setup = time.perf_counter()
        if fluid_name == "cpa6":
            results[label] = cpa_assembly_measure(local, shape, hbm_peak, relperm, timed)
            torch.cuda.empty_cache()
            continue
        else:
            grid, P, z = synth.natural_case(0, nx=shape[0], ny=shape[1], nz=shape[2])
            fluid = make_fluid()
            temperature = 353.15
            scale = 1.0
        ctx = Context(fluid, device=local)
        nat = NaturalAssembler(ctx, grid, 864.0, temperature, relperm)
        # cells whose P-T-z flash the reference cannot converge (a few per
        # million) take a converged cell's inputs, so the initial state exists
        fl = CubicThreePhaseFlash(fluid, device=local)
        st = fl.flash(P, np.full(grid.ncell, temperature), np.ascontiguousarray(z.T),
                      precision=abi.PRECISION_FP64_STAGED)["status"].cpu().numpy()
        bad, good = np.where(st != 0)[0], np.where(st == 0)[0]
        P, z = P.copy(), z.copy()
        P[bad], z[bad] = P[good[:bad.size]], z[good[:bad.size]]
        primary, ps = nat.initialize_from_ptz(P, z)
        nat.refresh_history(primary, ps)
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t_setup
        cur_np = synth.perturb_natural_state(primary.cpu().numpy(), ps.cpu().numpy(), fluid.nc, 11, scale)
        cur = torch.as_tensor(cur_np, device=primary.device)
        F = torch.empty_like(cur)
        vals = torch.empty(nat.nnzb, nat.B, nat.B, dtype=torch.float64, device=primary.device)
        work_p, work_s = cur.clone(), ps.clone()

        def update():
            work_p.copy_(cur)
            work_s.copy_(ps)
            return nat.update_state_with_report(work_p, work_s)

        def newton():
            update()
            nat.form_function(cur, ps, out=F)
            nat.assemble_jacobian(cur, ps, values=vals)

        n_rep = reps if grid.ncell <= 10000 else 1
        newton()   # warm-up
        torch.cuda.synchronize()
        t_update = sorted(timed(update) for _ in range(n_rep))
        t_res = sorted(timed(lambda: nat.form_function(cur, ps, out=F)) for _ in range(max(n_rep, 3)))
        t_jac = sorted(timed(lambda: nat.assemble_jacobian(cur, ps, values=vals)) for _ in range(max(n_rep, 3)))
        t_newton = sorted(timed(newton) for _ in range(n_rep))
        # both update forms: every stability test and reflash on the batched
        # staged kernels, or inside each cell's own thread / warp
        nat.set_update_mode("staged")
        t_update_staged = sorted(timed(update) for _ in range(n_rep))
        nat.set_update_mode("per_cell")
        t_update_per_cell = timed(update)
        nat.set_update_mode("auto")
        rc, rep = update()
        jac_bytes = nat.nnzb * nat.B * nat.B * 8 + grid.ncell * nat.B * 8
        jac_ms = t_jac[len(t_jac) // 2]
        host_vals = torch.empty(vals.shape, dtype=vals.dtype, pin_memory=True)
        d2h_ms = timed(lambda: host_vals.copy_(vals, non_blocking=True))
        entry = {
            "cells": grid.ncell, "faces": int(grid.nfaces), "block": nat.B, "blocks": nat.nnzb,
            "fluid": "six-component PR-CPA (4C water, CO2 acceptor)" if fluid_name == "cpa6"
                     else "H2O/CO2/nC10 PR", "temperature_K": temperature,
            "setup_s": setup_s,
            "newton_eval_ms": {"p50": t_newton[len(t_newton) // 2], "max": t_newton[-1], "reps": n_rep},
            "cell_evals_per_s": grid.ncell / (t_newton[len(t_newton) // 2] * 1e-3),
            "update_ms": t_update[len(t_update) // 2],
            "update_form_auto": "staged" if grid.ncell >= 148 * 256 else "per-cell (warp per cell)",
            "update_ms_staged_form": t_update_staged[len(t_update_staged) // 2],
            "update_ms_per_cell_form": t_update_per_cell,
            "residual_ms": t_res[len(t_res) // 2],
            "jacobian_ms": jac_ms,
            "baij_device_to_host_ms": d2h_ms,
            "update_committed": rc == 0,
            "stable_reduced_cells": int(rep.stable_reduced_cells),
            "jacobian_roofline": {"bound": "hbm", "bytes_per_launch": jac_bytes,
                                  "achieved": jac_bytes / (jac_ms * 1e-3) / 1e9, "unit": "GB/s",
                                  "peak": hbm_peak,
                                  "frac": (jac_bytes / (jac_ms * 1e-3) / 1e9 / hbm_peak) if hbm_peak else None},
        }
        if with_cpu and label == "60x20x1":
            try:
                from oracle import ref
                if ref.available():
                    cpu = {}
                    p0, s0 = primary.cpu().numpy(), ps.cpu().numpy()
                    for threads in (1, os.cpu_count() or 1):
                        oracle = ref.Natural(fluid, grid, 864.0, temperature, relperm)
                        oracle.set_threads(threads)
                        oracle.set_history(p0, s0)
                        t0 = time.perf_counter()
                        oracle.update_state(cur_np, s0)
                        oracle.residual(cur_np, s0)
                        oracle.jacobian(cur_np, s0)
                        dt = time.perf_counter() - t0
                        cpu[f"{threads}_threads"] = {"newton_eval_ms": dt * 1e3, "cell_evals_per_s": grid.ncell / dt}
                    entry["cpu_reference"] = {**cpu, "kind": "reference",
                                              "what": "the reference's updatePhaseState / residual / Jacobian "
                                                      "loops (oracle/_ref) on the same state, one kernel per thread"}
            except Exception as ex:
                entry["cpu_reference"] = {"error": str(ex)}
        results[label] = entry
        del nat, ctx, fl, vals, host_vals
        torch.cuda.empty_cache()
    return results


def serving_measure(local: int, n_requests: int, rate: float = 20.0, slots: int = 4):
    """The request loop (nonenone_b200.serving) over a Poisson stream: each
    request one flash + assembly job (new model: per-cell P-T-z flash, history,
    residual, BAIJ Jacobian; repeat iteration of a resident model, 30 %:
    warm-started phase-state update, residual, Jacobian); nc 3-8, EOS 50 / 30 /
    20 % PR / SW / PR-CPA, 150 GB admission budget, 4 slots.  Cell counts are
    log-uniform in [1e3, 1e4] (the benchmark's [1e3, 1e6] scaled down so a
    run of PR-CPA and SW initialisations stays within the bench's minutes)."""
    from nonenone_b200 import serving
    reqs = serving.poisson_requests(n_requests, rate=rate, seed=5, cells=(1.0e3, 1.0e4))
    ex = serving.NaturalExecutor(device=local, slots=slots)
    # build the fluids' contexts before the clock starts
    for r in reqs:
        ex._context(r.nc, r.eos, 0)
    out = serving.ServingLoop(ex, slots=slots, hbm_budget=150.0e9).run(reqs)
    stats = serving.summarize(out)
    stats.update({"arrival_rate_req_per_s": rate, "slots": slots, "hbm_budget_bytes": 150.0e9,
                  "cells": "log-uniform [1e3, 1e4]", "repeat_fraction": 0.3,
                  "errors": [o.error for o in out if o.error][:3]})
    return stats


def models_measure(local: int, nmodels: int, cells, seed: int = 21, precision: int | None = None):
    """The uneven multi-model batch: `nmodels` models, cell counts log-uniform
    on `cells`, nc uniform over {3,4,5,6,8}, EOS uniform over PR / SW / PR-CPA,
    P/T/z drawn as on the hydrostatic benchmark grid (synth.model_points).
    One ModelBatch (per-nc groups, per-point fluids, one captured CUDA graph,
    launch shapes from its autotuner) against the same models flashed by
    separate per-model calls back to back on one stream; both device-event
    timed, answers compared label for label."""
    import torch
    from nonenone_b200 import abi, synth
    from nonenone_b200.flash import CubicThreePhaseFlash
    from nonenone_b200.fluids import model_fluid
    from nonenone_b200.models import ModelBatch
    if precision is None:
        precision = abi.PRECISION_FP64_STAGED
    dev = torch.device("cuda", local)
    specs = synth.model_batch_specs(nmodels, cells, seed=seed)
    ins = []
    for k, (nc, eos, n) in enumerate(specs):
        P, T, z, sal = synth.model_points(nc, n, seed=1000 + k)
        t = [torch.as_tensor(x, device=dev) for x in (P, T, z)]
        if eos == "sw":
            t.append(torch.as_tensor(sal, device=dev))
        ins.append(tuple(t))
    total = sum(n for _, _, n in specs)
    mb = ModelBatch([model_fluid(nc, eos) for nc, eos, _ in specs], [n for _, _, n in specs], device=local)
    t0 = time.perf_counter()
    chosen = mb.tune(ins, precision, sample_points=512)
    torch.cuda.synchronize()
    tune_s = time.perf_counter() - t0
    outs = mb.allocate()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    mb.flash(ins, precision, outs)   # capture
    torch.cuda.synchronize()
    grouped_ms = timed(lambda: mb.flash(ins, precision, outs))
    evals = mb.eos_eval_count()
    check_words = mb.self_check()
    ctxs = [CubicThreePhaseFlash(model_fluid(nc, eos), device=local) for nc, eos, _ in specs]
    souts = [c.allocate(n) for c, (_, _, n) in zip(ctxs, specs)]

    def separate():
        for c, inp, o, (_, _, n) in zip(ctxs, ins, souts, specs):
            if n:
                c.flash(inp[0], inp[1], inp[2], salinity=inp[3] if len(inp) > 3 else None,
                        precision=precision, out=o)

    separate()
    torch.cuda.synchronize()
    separate_ms = timed(separate)
    mismatch = sum(int((outs[k]["presence"] != souts[k]["presence"]).sum().item()) +
                   int((outs[k]["status"] != souts[k]["status"]).sum().item()) for k in range(len(specs)))
    by_eos = {}
    for nc, eos, n in specs:
        by_eos[eos] = by_eos.get(eos, 0) + n
    groups = sorted({nc for nc, _, n in specs if n > 0})
    res = {
        "models": nmodels, "cells": total, "cells_by_eos": by_eos,
        "scaled_from": ("the benchmark's 256 models of 1e4-5e5 cells (about 3e7 cells); Soreide-Whitson "
                        "and PR-CPA models at nc 6-8 flash at ~0.5-1.4 k cells/s on their own at these "
                        "P/T/z, so the set is scaled down to keep the bench within minutes"),
        "cell_range": f"log-uniform [{cells[0]:.0e}, {cells[1]:.0e}]",
        "component_counts": groups,
        "grouped": {"ms": grouped_ms, "cell_evals_per_s": total / (grouped_ms * 1e-3),
                    "eos_evals_per_cell": evals / max(total, 1), "graph": "one captured CUDA graph",
                    "kernel_launches": sum(staged_launches("fp64_staged", sw=any(e == "sw" and c == nc and n > 0
                                                                                 for c, e, n in specs)) + 2
                                           for nc in groups),
                    "self_check": {"queue_bound": check_words[0], "spin_guard": check_words[1]}},
        "separate": {"ms": separate_ms, "cell_evals_per_s": total / (separate_ms * 1e-3),
                     "kernel_launches": sum(staged_launches("fp64_staged", sw=e == "sw") for _, e, n in specs if n)},
        "grouped_over_separate": separate_ms / grouped_ms,
        "label_or_status_mismatch_vs_separate": mismatch,
        "autotuner": {"chosen_blocks_per_sm": {str(nc): {"lane": v[0], "warp": v[1]} for nc, v in chosen.items()},
                      "seconds": tune_s, "sample_points_per_nc": 512},
    }
    mb.close()
    return res


def cpa_assembly_measure(local, shape, hbm_peak, relperm, timed, block=(20, 20)):
    """Residual + BAIJ Jacobian assembly of one Newton iterate on the
    200x200x50 hydrostatic grid with the six-component PR-CPA fluid (B = 19),
    and the device-to-host copy of the BAIJ values.  The initial state is the
    P-T-z flash of a block x nz column of the grid, tiled over the x-y plane
    (P depends on depth only; a full 2,000,000-cell CPA flash would dominate
    the run), then perturbed; porosity, permeability and the iterate are the
    full grid's own."""
    import torch
    from nonenone_b200 import abi, synth
    from nonenone_b200.flash import Context
    from nonenone_b200.fluids import make_cpa_six
    from nonenone_b200.natural import NaturalAssembler
    t0 = time.perf_counter()
    nx, ny, nz = shape
    grid, P, z, depth = synth.natural_case_hydrostatic(3, nx=nx, ny=ny, nz=nz)
    fluid = make_cpa_six()
    temperature = 373.15 + 0.03 * float(np.median(depth))
    bx, by = block
    sub, Ps, zs, _ = synth.natural_case_hydrostatic(3, nx=bx, ny=by, nz=nz)
    ctx = Context(fluid, device=local)
    small = NaturalAssembler(ctx, sub, 864.0, temperature, relperm)
    p_blk, s_blk = small.initialize_from_ptz(Ps, zs)
    idx = ((grid.k * by + grid.j % by) * bx + grid.i % bx).astype(np.int64)
    dev = p_blk.device
    primary = p_blk[torch.as_tensor(idx, device=dev)].contiguous()
    ps = s_blk[torch.as_tensor(idx, device=dev)].contiguous()
    del small
    nat = NaturalAssembler(ctx, grid, 864.0, temperature, relperm)
    nat.refresh_history(primary, ps)
    # the assembly at the accepted state (any perturbation of 2,000,000 PR-CPA
    # cells puts some cell where the reference's association solve gives up,
    # which is a domain error of the whole evaluation)
    cur = primary
    F = torch.empty_like(cur)
    vals = torch.empty(nat.nnzb, nat.B, nat.B, dtype=torch.float64, device=dev)
    nat.form_function(cur, ps, out=F)
    nat.assemble_jacobian(cur, ps, values=vals)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    t_res = sorted(timed(lambda: nat.form_function(cur, ps, out=F)) for _ in range(3))
    t_jac = sorted(timed(lambda: nat.assemble_jacobian(cur, ps, values=vals)) for _ in range(3))
    host_vals = torch.empty(vals.shape, dtype=vals.dtype, pin_memory=True)
    d2h_ms = timed(lambda: host_vals.copy_(vals, non_blocking=True))
    jac_bytes = nat.nnzb * nat.B * nat.B * 8 + grid.ncell * nat.B * 8
    jac_ms = t_jac[1]
    out = {
        "cells": grid.ncell, "faces": int(grid.nfaces), "block": nat.B, "blocks": nat.nnzb,
        "fluid": "six-component PR-CPA (4C water, CO2 acceptor)", "temperature_K": temperature,
        "initial_state": f"P-T-z flash of a {bx}x{by}x{nz} column tiled over the x-y plane; assembled at that "
                         f"accepted state",
        "setup_s": setup_s,
        "residual_ms": t_res[1], "jacobian_ms": jac_ms,
        "newton_assembly_ms": t_res[1] + jac_ms,
        "cell_evals_per_s": grid.ncell / ((t_res[1] + jac_ms) * 1e-3),
        "baij_device_to_host_ms": d2h_ms, "baij_bytes": vals.numel() * 8,
        "jacobian_roofline": {"bound": "hbm", "bytes_per_launch": jac_bytes,
                              "achieved": jac_bytes / (jac_ms * 1e-3) / 1e9, "unit": "GB/s", "peak": hbm_peak,
                              "frac": (jac_bytes / (jac_ms * 1e-3) / 1e9 / hbm_peak) if hbm_peak else None},
    }
    # the reference's residual + Jacobian loops on all host threads, over the
    # flashed column (its own grid, the same accepted state), per cell
    try:
        from oracle import ref
        threads = os.cpu_count() or 1
        o = ref.Natural(fluid, sub, 864.0, temperature, relperm)
        o.set_threads(threads)
        pb, sb = p_blk.cpu().numpy(), s_blk.cpu().numpy()
        o.set_history(pb, sb)
        tc = time.perf_counter()
        o.residual(pb, sb)
        o.jacobian(pb, sb)
        cpu_s = time.perf_counter() - tc
        out["cpu_reference"] = {"threads": threads, "cells": sub.ncell, "newton_assembly_ms": cpu_s * 1e3,
                                "cell_evals_per_s": sub.ncell / cpu_s, "kind": "reference",
                                "what": f"the reference's residual and Jacobian loops (oracle/_ref) on the "
                                        f"{bx}x{by}x{nz} column at its accepted state"}
    except Exception as ex:   # the compiled reference is test infrastructure; report, do not fail
        out["cpu_reference"] = {"error": str(ex)}
    del nat, vals, host_vals
    return out


def next_offset(off: int, m: int, n: int) -> int:
    """Start of the next m-point sample of an n-point workload: the samples
    rotate through the workload and wrap; a sample of the whole workload
    (m >= n) always starts at 0."""
    if m >= n:
        return 0
    return (off + m) % (n - m + 1)


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    from nonenone_b200 import synth
    from nonenone_b200.fluids import make_fluid
    from oracle import ref
    fluid = make_fluid()
    n_points = args.points
    if n_points == N_POINTS:
        # the GPU arm's first batch: label mixture + near-boundary slice
        P, T, z = synth.benchmark_points(n_points, boundary_slice(), seed=1)
    else:
        P, T, z = synth.flash_points(n_points, seed=1)
    threads = os.cpu_count() or 1
    # each step is a bounded, rotating sample of the workload sized so the
    # whole --steps/--warmup run stays within a few minutes
    probe = min(256, n_points)
    t0 = time.perf_counter()
    ref.flash_batch(fluid, P[:probe], T[:probe], z[:, :probe], threads=1)
    per_point = (time.perf_counter() - t0) / probe
    m = int(min(n_points, max(threads * 32, 8.0 * threads / max(per_point, 1e-7))))
    off = 0
    for _ in range(args.warmup):
        sl = slice(off, off + m)
        ref.flash_batch(fluid, P[sl], T[sl], z[:, sl], threads=threads)
        off = next_offset(off, m, n_points)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sl = slice(off, off + m)
        ref.flash_batch(fluid, P[sl], T[sl], z[:, sl], threads=threads)
        off = next_offset(off, m, n_points)
    dt = time.perf_counter() - t0
    rate = m * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "points_per_step": m, "eos": "PR", "nc": NC},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{m} of the {n_points} workload points per step (rotating), "
                                   f"{threads} threads, one CubicThreePhaseFlash each"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


FORMS = ("fp64", "fp64_staged", "mixed")


def staged_launches(precision_name: str, sw: bool = False) -> int:
    """Kernels one batch launches: the plain FP64 form one; the staged forms
    start, 8 rounds x 8, recovery 1 (5), recovery 2 (3 x 2), the recovery
    kernel (SW: the allocation queue and seed kernels, then the recovery
    kernel in two passes around the role-permutation kernel), the
    continuation anchors, select and check (+ for the mixed form its
    FP32 trial phase before each of the 11 trial launches, and the polish)."""
    if precision_name == "fp64":
        return 1
    recovery = 5 if sw else 1
    return 1 + 8 * 8 + 5 + 3 * 2 + recovery + 1 + 1 + 1 + (12 if precision_name == "mixed" else 0)


def form_error(out, ref_out):
    """Label / status differences and largest relative value differences of a
    flash answer against another on the same batch (both device dicts)."""
    a = {k: v.cpu().numpy() for k, v in out.items()}
    b = {k: v.cpu().numpy() for k, v in ref_out.items()}
    same = (a["status"] == b["status"]) & (a["presence"] == b["presence"])
    ok = same & (b["status"] == 0)
    err = {"points": int(a["status"].size), "label_or_status_mismatch": int((~same).sum())}
    present = np.stack([(b["presence"] >> p) & 1 for p in range(3)]).astype(bool) & ok
    for key in ("beta", "composition", "saturation", "compressibility", "k_gas_oil", "k_water_oil"):
        x, y = a[key], b[key]
        if key in ("saturation", "compressibility"):
            x, y = x[present], y[present]
        else:
            x, y = x[..., ok], y[..., ok]
        fin = np.isfinite(y)
        e = np.abs(x - y)[fin] / np.maximum(1.0, np.abs(y[fin]))
        err[key + "_max_rel"] = float(e.max()) if e.size else 0.0
    return err


def residual_summary(eos, P, T, out, salinity=None):
    import torch
    from nonenone_b200.flash import fugacity_residual
    r = fugacity_residual(eos, P, T, out, salinity=salinity)
    fin = r[torch.isfinite(r)]
    if not fin.numel():
        return {"fugacity_residual_max": None}
    return {"fugacity_residual_max": float(fin.max()),
            "fugacity_residual_p99": float(torch.quantile(fin[:1 << 24], 0.99)),
            "fugacity_residual_above_1e-10": int((fin > 1e-10).sum()),
            "multiphase_points": int(fin.numel())}


def run_gpu(args):
    import torch
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from nonenone_b200 import abi, synth
    from nonenone_b200.fluids import make_fluid
    from nonenone_b200.flash import CubicEquationOfState, CubicThreePhaseFlash
    from nonenone_b200.lib import load

    prec_of = {"fp64": abi.PRECISION_FP64, "fp64_staged": abi.PRECISION_FP64_STAGED,
               "mixed": abi.PRECISION_MIXED}
    headline = args.precision
    precision = prec_of[headline]
    fluid = make_fluid()
    M = max(1, args.inflight)
    dev = torch.device("cuda", local)
    main = torch.cuda.current_stream()

    # the benchmark batch: the label mixture plus the 5 % near-boundary slice
    boundary = boundary_slice()
    nb = boundary[0].shape[0]
    slots = []
    for m in range(M):
        fl = CubicThreePhaseFlash(fluid, device=local)
        P, T, z = synth.benchmark_points(N_POINTS, boundary, seed=1 + 1000 * rank + m)
        slots.append(dict(
            fl=fl, stream=torch.cuda.Stream(device=dev),
            P=torch.tensor(P, device=dev), T=torch.tensor(T, device=dev),
            z=torch.tensor(z, device=dev), out=fl.allocate(N_POINTS), host=(P, T, z)))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def run_steps(nsteps, prec, e0, e1, inflight=M):
        e0.record(main)
        for sl in slots[:inflight]:
            sl["stream"].wait_event(e0)
        for k in range(nsteps):
            sl = slots[k % inflight]
            sl["fl"].flash(sl["P"], sl["T"], sl["z"], out=sl["out"], precision=prec, stream=sl["stream"])
        for sl in slots[:inflight]:
            ev = torch.cuda.Event()
            ev.record(sl["stream"])
            main.wait_event(ev)
        e1.record(main)

    def timed_rate(prec, nsteps, inflight):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        run_steps(nsteps, prec, a, b, inflight)
        torch.cuda.synchronize()
        return N_POINTS * nsteps / (a.elapsed_time(b) * 1e-3)

    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    run_steps(max(args.warmup, 1), precision, w0, w1)
    barrier()
    lat = []
    for _ in range(args.latency_reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(main)
        slots[0]["fl"].flash(slots[0]["P"], slots[0]["T"], slots[0]["z"], out=slots[0]["out"],
                             precision=precision, stream=main)
        b.record(main)
        torch.cuda.synchronize()
        lat.append(a.elapsed_time(b))
    evals_per_batch = slots[0]["fl"].eos_eval_count()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier()
        run_steps(args.steps, precision, e0, e1)
        barrier()
    total_ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = N_POINTS * world * args.steps / (total_ms * 1e-3)
    self_check = slots[0]["fl"].self_check() if precision != abi.PRECISION_FP64 else (0, 0)

    # --- e2e: pinned host inputs -> public entry point -> pinned host results ----
    for sl in slots:
        P, T, z = sl["host"]
        sl["hP"] = torch.from_numpy(P).pin_memory()
        sl["hT"] = torch.from_numpy(T).pin_memory()
        sl["hz"] = torch.from_numpy(z).pin_memory()
        sl["hout"] = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in sl["out"].items()}
    h2d = N_POINTS * (2 + NC) * 8
    d2h = sum(t.numel() * t.element_size() for t in slots[0]["hout"].values())

    def e2e_launch(k):
        sl = slots[k % M]
        st = sl["stream"]
        with torch.cuda.stream(st):
            sl["P"].copy_(sl["hP"], non_blocking=True)
            sl["T"].copy_(sl["hT"], non_blocking=True)
            sl["z"].copy_(sl["hz"], non_blocking=True)
        sl["fl"].flash(sl["P"], sl["T"], sl["z"], out=sl["out"], precision=precision, stream=st)
        with torch.cuda.stream(st):
            for key, t in sl["out"].items():
                sl["hout"][key].copy_(t, non_blocking=True)

    e2e_steps = max(1, args.steps)
    barrier()
    t0 = time.perf_counter()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(main)
    for sl in slots:
        sl["stream"].wait_event(a)
    for k in range(e2e_steps):
        e2e_launch(k)
    for sl in slots:
        ev = torch.cuda.Event()
        ev.record(sl["stream"])
        main.wait_event(ev)
    b.record(main)
    barrier()
    e2e_s = max(time.perf_counter() - t0, a.elapsed_time(b) * 1e-3)
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = N_POINTS * world * e2e_steps / e2e_s

    # --- the other forms on the same batches, accuracy of each -------------------
    forms = None
    sw_half = None
    if rank == 0 and not args.no_forms:
        eos = CubicEquationOfState(fluid, device=local)
        s0 = slots[0]
        ref_out = s0["fl"].flash(s0["P"], s0["T"], s0["z"], precision=abi.PRECISION_FP64_STAGED)
        torch.cuda.synchronize()
        forms = {}
        for name in FORMS:
            pr = prec_of[name]
            if name == headline:
                rate = value / world
            else:
                inflight = min(2, M)
                timed_rate(pr, inflight, inflight)   # warm-up of the form
                rate = timed_rate(pr, inflight, inflight)
            o = s0["fl"].flash(s0["P"], s0["T"], s0["z"], precision=pr)
            entry = {"flashes_per_s": rate, **residual_summary(eos, s0["P"], s0["T"], o)}
            if name != "fp64_staged":
                entry["error_vs_fp64_staged"] = form_error(o, ref_out)
            forms[name] = entry
        base = forms["fp64"]["flashes_per_s"]
        for name in FORMS:
            forms[name]["vs_plain_fp64"] = forms[name]["flashes_per_s"] / base
        # the Soreide-Whitson half: the same mixture with salinity ~ U[0,2] mol/kg
        swf = make_fluid(eos_model=abi.EOS_SW)
        swl = CubicThreePhaseFlash(swf, device=local)
        swe = CubicEquationOfState(swf, device=local)
        n_sw = N_POINTS // 16
        Pw, Tw, zw, sal = synth.flash_points(n_sw, seed=2 + 1000 * rank, salinity=True)
        dPw, dTw, dzw, dsw = (torch.tensor(x, device=dev) for x in (Pw, Tw, zw, sal))
        sw_half = {"workload": f"{n_sw} points of the label mixture (a sixteenth of the PR batch: the SW "
                               f"recoveries make a point ~16x the work), Soreide-Whitson, salinity ~ U[0,2]"}
        sw_ref = None
        for name in ("fp64_staged", "mixed"):
            pr = prec_of[name]
            outw = swl.allocate(n_sw)
            swl.flash(dPw, dTw, dzw, salinity=dsw, precision=pr, out=outw)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(main)
            swl.flash(dPw, dTw, dzw, salinity=dsw, precision=pr, out=outw)
            b.record(main)
            torch.cuda.synchronize()
            sw_half[name] = {"flashes_per_s_one_batch": n_sw / (a.elapsed_time(b) * 1e-3),
                             **residual_summary(swe, dPw, dTw, outw, salinity=dsw)}
            if sw_ref is None:
                sw_ref = {k: v.clone() for k, v in outw.items()}
            else:
                sw_half[name]["error_vs_fp64_staged"] = form_error(outw, sw_ref)

    # --- roofline ---------------------------------------------------------------
    lib = load()
    import ctypes as C
    fp64 = C.c_double()
    fp32 = C.c_double()
    lib.nz_diag_fma_peak(local, C.byref(fp64), C.byref(fp32))
    step_s = total_ms * 1e-3 / args.steps
    flops = evals_per_batch * f_eos(NC)
    achieved = flops / step_s / 1e12
    peak = fp64.value
    status = slots[0]["out"]["status"].cpu().numpy()
    presence = slots[0]["out"]["presence"].cpu().numpy()

    serving_stats = None
    if rank == 0 and args.serving_requests > 0:
        serving_stats = serving_measure(local, args.serving_requests, slots=args.serving_slots)

    multi_model = None
    if rank == 0 and args.models > 0:
        lo, hi = (float(v) for v in args.model_cells.split(","))
        multi_model = models_measure(local, args.models, (lo, hi))

    natural = None
    if rank == 0 and not args.no_natural:
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
                hbm_peak = float(json.load(fh)["hbm_gbs"])
        except Exception:
            hbm_peak = 6650.0
        natural = natural_measure(local, 5, hbm_peak, not args.no_cpu_baseline, not args.no_cpa_natural)

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            try:
                from oracle import ref
                if ref.available():
                    P, T, z = slots[0]["host"]
                    cpu = cpu_reference_rate(fluid, P, T, z)
            except Exception as ex:   # the baseline must not mask the GPU number
                cpu = {"value": None, "error": str(ex)}
        lat_sorted = sorted(lat)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if precision == abi.PRECISION_MIXED else "f64",
            "data": "synthetic (seeded: nonenone_b200.synth label mixture + 5 % near-boundary slice)",
            "config": {"workload": WORKLOAD,
                       "points_per_batch": N_POINTS, "eos": "PR", "nc": NC,
                       "precision": headline, "batches_in_flight": M,
                       "near_boundary_points": nb,
                       "mixture": ("95 % a label-free proposal mixture drawn to ~40/40/20 % single/two/three-phase "
                                   "by the reference label: 45 % z_H2O ~ U[0, 5e-4] with (CO2, nC10) ~ Dir(1, 1) "
                                   "in the box's P/T; 32 % the box itself (P ~ U[5, 40] MPa, T ~ U[303, 423] K, "
                                   "z ~ Dir(2, 1, 1)); 23 % a three-phase proposal outside the box's z law "
                                   "(P ~ U[5, 12] MPa, T ~ U[340, 423] K, z ~ Dir(2, 2, 0.6)); + 5 % within "
                                   "5e-6 relative of a pressure where a phase appears"),
                       "l2": f"not flushed: {M} distinct input sets of 42 MB and output sets of "
                             f"{d2h / 1e6:.0f} MB per batch in flight exceed the 126 MB L2",
                       "label_mix": {"single": float(np.isin(presence, [1, 2, 4]).mean()),
                                     "two": float(np.isin(presence, [3, 5, 6]).mean()),
                                     "three": float((presence == 7).mean()),
                                     "failed": float((status != 0).mean())}},
            "latency_ms": {"p50": float(np.percentile(lat_sorted, 50)),
                           "p99": float(np.percentile(lat_sorted, 99)), "samples": len(lat_sorted),
                           "what": "one isolated 1,048,576-point batch of the headline form, CUDA events"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "entry_point": "nz_flash_batch on pinned-host-fed device buffers, copies on the "
                                   "batch's stream inside the timed region"},
            "roofline": {"bound": "fp64",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": None,
                         "peak_source": "measured on this GPU by nz_diag_fma_peak (FMA chains); "
                                        "not in MEASURED_PEAKS.json",
                         "flops_per_batch": flops,
                         "eos_evals_per_flash": float(evals_per_batch / N_POINTS),
                         "flops_convention": "executed single-phase EOS evaluations x F_eos(nc), "
                                             "F_eos(nc) = 2 nc^2 + 13 nc + 50",
                         "frac_with_transcendentals": ((evals_per_batch * (f_eos(NC) + 20 * (NC + 7))
                                                        / step_s / 1e12) / peak) if peak else None,
                         "transcendental_convention": "the nc + 7 log / exp / sqrt calls of an EOS "
                                                      "evaluation counted as 20 FP64 operations each",
                         "kernel": "flash pipeline (all kernels of one batch)"},
            "gpu_launches": args.steps * staged_launches(headline),
            "self_check": {"queue_bound": self_check[0], "spin_guard": self_check[1]},
            "forms": forms,
            "sw_half": sw_half,
            "clocks": clocks.summary(),
            "fp32_fma_peak_tflops": fp32.value,
            "cpu_baseline": cpu,
            "natural": natural,
            "serving": serving_stats,
            "multi_model": multi_model,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nz", choices=["nz", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "fp64_staged", "mixed"],
                    help="headline form (the others are measured beside it unless --no-forms)")
    ap.add_argument("--latency-reps", type=int, default=8)
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the other precision forms and the Soreide-Whitson half")
    ap.add_argument("--inflight", type=int, default=4)
    ap.add_argument("--points", type=int, default=N_POINTS,
                    help="workload size of the reference arm (the benchmark's is 1,048,576)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-natural", action="store_true",
                    help="skip the Natural Newton-evaluation measurements")
    ap.add_argument("--serving-requests", type=int, default=24,
                    help="requests of the serving-loop measurement (0 skips it)")
    ap.add_argument("--serving-slots", type=int, default=8,
                    help="concurrent request slots of the serving loop")
    ap.add_argument("--models", type=int, default=32,
                    help="models of the uneven multi-model batch measurement (0 skips it)")
    ap.add_argument("--model-cells", default="100,1000",
                    help="cell-count range lo,hi (log-uniform) of the multi-model batch")
    ap.add_argument("--no-cpa-natural", action="store_true",
                    help="skip the six-component PR-CPA Natural grid")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
