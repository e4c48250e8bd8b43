"""Generate the committed golden fixtures of tests/golden/ from the reference.

Run in a container where the reference tree is present and oracle/_ref is
built (python -m nonenone_b200.build --oracle).  Every array comes from the
reference's own FP64 C++ (oracle/_ref/libnzref.so); the inputs are seeded
(nonenone_b200.synth), so the fixtures can be regenerated bit for bit.

  flash_pr_nc3.npz  2048 points of the batched-flash mixture, PR
  flash_sw_nc3.npz  1024 points, Soreide-Whitson, salinity ~ U[0,2]
  flash_pr_nc6.npz  512 points, six components, PR
Each holds the inputs, the full nz_flash_out record, and for converged
points the stability trial sums of the missing phases of the final state
(|trialSum - 1| is the distance to the phase boundary used to exclude
boundary points from label comparisons).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from nonenone_b200 import abi, synth  # noqa: E402
from nonenone_b200.fluids import SIX_COMPONENT, make_fluid  # noqa: E402
from oracle import ref  # noqa: E402


def boundary_distance(fluid, P, T, z, out, salinity=None):
    """min over missing phases of |trialSum - 1| for converged points (inf otherwise)."""
    n = P.shape[0]
    dist = np.full(n, np.inf)
    ok = (out["status"] == abi.FLASH_CONVERGED) & (out["presence"] != 7) & (out["presence"] != 0)
    idx = np.where(ok)[0]
    if idx.size == 0:
        return dist
    st = ref.stability_batch(fluid, P[idx], T[idx], z[:, idx], out["presence"][idx],
                             out["composition"][:, :, idx],
                             None if salinity is None else salinity[idx], threads=8)
    ts = st["trial_sum"]
    for k, i in enumerate(idx):
        pres = out["presence"][i]
        d = [abs(ts[p, k] - 1.0) for p in range(3) if not (pres >> p) & 1]
        dist[i] = min(d) if d else np.inf
    return dist


def make(name, fluid, P, T, z, salinity=None):
    out = ref.flash_batch(fluid, P, T, z, salinity=salinity, threads=8)
    dist = boundary_distance(fluid, P, T, z, out, salinity)
    arrays = dict(P=P, T=T, z=z, tpd_distance=dist, **out)
    if salinity is not None:
        arrays["salinity"] = salinity
    np.savez_compressed(os.path.join(HERE, name), **arrays)
    labels = np.bincount(out["presence"], minlength=8)
    print(name, "status", np.bincount(out["status"], minlength=5), "presence", labels)


def main():
    if not ref.available():
        raise SystemExit("oracle/_ref is not built")
    pr = make_fluid()
    P, T, z = synth.flash_points(2048, seed=101)
    make("flash_pr_nc3.npz", pr, P, T, z)
    sw = make_fluid(eos_model=abi.EOS_SW)
    P, T, z, s = synth.flash_points(1024, seed=102, salinity=True)
    make("flash_sw_nc3.npz", sw, P, T, z, s)
    six = make_fluid(SIX_COMPONENT)
    rng = np.random.default_rng(103)
    n = 512
    P = rng.uniform(5e6, 40e6, n)
    T = rng.uniform(303.0, 423.0, n)
    z = np.ascontiguousarray(rng.dirichlet([4, 2, 1, 1, 1, 1], n).T)
    make("flash_pr_nc6.npz", six, P, T, z)


if __name__ == "__main__":
    main()
