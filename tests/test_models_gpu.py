"""Uneven multi-model batches on the GPU: every model's answer from the shared
graph-captured launch equals its own CubicThreePhaseFlash.flash run (the same
per-point code, so bit for bit), for PR / SW / PR-CPA models of every compiled
component count, on the first call (capture), on a replay, after the
autotuner, and in the mixed form."""
import numpy as np
import pytest

from nonenone_b200 import abi, synth
from nonenone_b200.fluids import model_fluid

pytestmark = pytest.mark.gpu

FIELDS = ("presence", "status", "beta", "saturation", "composition", "compressibility",
          "molar_density", "k_gas_oil", "k_water_oil", "iterations")


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    return torch


def _specs():
    # every (nc, eos) pair once, uneven sizes, plus one empty model
    specs = []
    sizes = [37, 300, 1200, 90, 2500, 640, 1, 777]
    k = 0
    for nc in synth.MODEL_NCS:
        for eos in synth.MODEL_EOS:
            specs.append((nc, eos, sizes[k % len(sizes)]))
            k += 1
    specs.append((3, "pr", 0))
    return specs


def _inputs(torch, specs):
    ins = []
    for k, (nc, eos, n) in enumerate(specs):
        P, T, z, sal = synth.model_points(nc, n, seed=100 + k)
        t = [torch.as_tensor(x, device="cuda") for x in (P, T, z)]
        if eos == "sw":
            t.append(torch.as_tensor(sal, device="cuda"))
        ins.append(tuple(t))
    return ins


def _solo(torch, specs, ins, precision):
    from nonenone_b200.flash import CubicThreePhaseFlash
    outs = []
    for (nc, eos, n), inp in zip(specs, ins):
        fl = CubicThreePhaseFlash(model_fluid(nc, eos))
        o = fl.allocate(n)
        if n:
            fl.flash(inp[0], inp[1], inp[2], salinity=inp[3] if len(inp) > 3 else None,
                     precision=precision, out=o)
        torch.cuda.synchronize()
        outs.append({k: v.cpu().numpy() for k, v in o.items()})
    return outs


def _same(specs, got, want, what):
    for k, ((nc, eos, n), g, w) in enumerate(zip(specs, got, want)):
        if n == 0:
            continue
        for f in FIELDS:
            a, b = g[f].cpu().numpy(), w[f]
            if f in ("saturation", "compressibility", "molar_density", "beta", "composition"):
                # absent phases carry no physical value; compare the present ones
                pres = np.stack([(w["presence"] >> p) & 1 for p in range(3)]).astype(bool)
                ok = (w["status"] == abi.FLASH_CONVERGED)
                mask = pres & ok
                if f == "composition":
                    mask = np.repeat(mask[:, None, :], nc, axis=1)
                a, b = a[mask], b[mask]
            elif f in ("k_gas_oil", "k_water_oil"):
                ok = w["status"] == abi.FLASH_CONVERGED
                a, b = a[:, ok], b[:, ok]
            assert np.array_equal(a, b), (what, k, nc, eos, f)


def test_models_equal_solo_runs(torch_cuda):
    torch = torch_cuda
    from nonenone_b200.models import ModelBatch
    specs = _specs()
    ins = _inputs(torch, specs)
    want = _solo(torch, specs, ins, abi.PRECISION_FP64_STAGED)
    mb = ModelBatch([model_fluid(nc, eos) for nc, eos, _ in specs], [n for _, _, n in specs])
    outs = mb.flash(ins, abi.PRECISION_FP64_STAGED)
    torch.cuda.synchronize()
    assert mb.self_check() == (0, 0)
    assert mb.eos_eval_count() > 0
    _same(specs, outs, want, "capture")
    # a replay of the captured graph into fresh outputs
    outs2 = mb.flash(ins, abi.PRECISION_FP64_STAGED)
    torch.cuda.synchronize()
    _same(specs, outs2, want, "replay")
    # the autotuner, then a new capture with the chosen shapes
    chosen = mb.tune(ins, abi.PRECISION_FP64_STAGED, sample_points=512)
    assert set(chosen) == set(synth.MODEL_NCS)
    for lane, warp in chosen.values():
        assert lane in (2, 4, 8, 16) and warp in (4, 8, 16)
    outs3 = mb.flash(ins, abi.PRECISION_FP64_STAGED)
    torch.cuda.synchronize()
    _same(specs, outs3, want, "tuned")
    mb.close()


def test_models_mixed_equal_solo_runs(torch_cuda):
    torch = torch_cuda
    from nonenone_b200.models import ModelBatch
    specs = [s for s in _specs() if s[1] != "sw"][:8]
    ins = _inputs(torch, specs)
    want = _solo(torch, specs, ins, abi.PRECISION_MIXED)
    mb = ModelBatch([model_fluid(nc, eos) for nc, eos, _ in specs], [n for _, _, n in specs])
    outs = mb.flash(ins, abi.PRECISION_MIXED)
    torch.cuda.synchronize()
    _same(specs, outs, want, "mixed")
    mb.close()


def test_models_reject_bad_arguments(torch_cuda):
    from nonenone_b200.lib import NzError
    from nonenone_b200.models import ModelBatch
    from nonenone_b200.fluids import make_fluid
    torch = torch_cuda
    no_water = make_fluid(("CO2", "C1", "nC10"))
    with pytest.raises(NzError):
        ModelBatch([no_water], [10])
    mb = ModelBatch([model_fluid(3, "pr")], [16])
    P, T, z, _ = synth.model_points(3, 16, seed=1)
    ins = [tuple(torch.as_tensor(x, device="cuda") for x in (P, T, z))]
    with pytest.raises(NzError):
        mb.flash(ins, abi.PRECISION_FP64)   # the plain form has no multi-model path
    with pytest.raises(NzError):
        mb.set_tuning(3, 0, 8)
    with pytest.raises(NzError):
        mb.tuning(6)
    mb.close()
