"""Generate the committed golden fixtures of tests/golden/ from the reference.

Run in a container where the reference tree is present and oracle/_ref is
built (python -m nonenone_b200.build --oracle).  Every array comes from the
reference's own FP64 C++ (oracle/_ref/libnzref.so); the inputs are seeded
(nonenone_b200.synth), so the fixtures can be regenerated bit for bit.

  flash_pr_nc3.npz  2048 points of the batched-flash mixture, PR
  flash_sw_nc3.npz  1024 points, Soreide-Whitson, salinity ~ U[0,2]
  flash_pr_nc6.npz  512 points, six components, PR
  flash_cpa_nc3.npz 1024 points, PR-CPA H2O/CO2/nC10 of the reference's 60x20 case
                    (4C water, CO2 one acceptor site: the single-donor path)
  flash_boundary_pr_nc3.npz  512 points next to a phase boundary
                    (synth.boundary_points with the reference's own labels): the
                    benchmark's near-boundary slice
  flash_boundary_sw_nc3.npz  256 such points, Soreide-Whitson, salinity ~ U[0,2]
  bench_boundary_pr_nc3.npz  the benchmark batch's near-boundary slice: 52,429
                    points (5 % of 1,048,576) of synth.boundary_points with the
                    reference's labels, inputs only; bench.py's GPU and reference
                    arms both take it (with the seeded label mixture)
  flash_continuation_pr_nc3.npz  192 points of the 1,048,576-point bench batch
                    (synth.flash_points(2**20, seed=1)) that reach the flash's last
                    fallback, the pressure continuation: 160 it rescues and 32 it
                    does not (RESCUED / FAILING below, found by scanning the batch
                    with this library's host-compiled solver with the continuation
                    switched off; only the choice of inputs comes from that scan)
Each holds the inputs, the full nz_flash_out record and, per point, the
distance of the reference's answer from a phase boundary in |TPD|
(tpd_distance; label comparisons exclude points below 1e-8).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from nonenone_b200 import abi, synth  # noqa: E402
from nonenone_b200.fluids import SIX_COMPONENT, make_cpa_h2o_co2_nc10, make_fluid  # noqa: E402
from oracle import ref  # noqa: E402


RESCUED = (
    187, 6787, 13970, 18453, 24723, 31078, 35682, 40026, 46128, 53689, 59326, 66687, 72474, 79984,
    88943, 94688, 99981, 103735, 113399, 119582, 124404, 128662, 135683, 142766, 146346, 154498,
    159325, 165215, 172093, 180023, 186797, 192793, 196887, 203081, 208501, 215626, 221446, 226343,
    232908, 238275, 243773, 251394, 256459, 263324, 269242, 273658, 280850, 288980, 293574, 301139,
    311750, 324317, 329344, 336068, 342327, 349748, 360265, 367787, 373327, 378244, 384988, 391227,
    396225, 403222, 408309, 413672, 419891, 425574, 433494, 438760, 447229, 454556, 462460, 468926,
    475364, 481293, 488043, 496799, 502081, 510908, 517967, 526451, 532261, 539193, 545951, 554840,
    561838, 568251, 573519, 578226, 584725, 593773, 599965, 605654, 613464, 624628, 630386, 636952,
    642374, 648314, 655679, 666178, 675259, 679812, 685584, 691809, 697421, 702248, 708573, 716886,
    724605, 732693, 738776, 744979, 752782, 755327, 759496, 766214, 776232, 783204, 791167, 798270,
    805079, 811706, 817122, 825149, 832689, 838979, 846530, 852708, 858652, 864868, 869100, 876423,
    882379, 888593, 893638, 899994, 905296, 910792, 916582, 922598, 930992, 933506, 938166, 944907,
    951407, 958644, 964378, 970957, 976391, 979846, 985294, 993079, 1000672, 1006878, 1012767,
    1018999, 1026386, 1033423,
)
FAILING = (
    2621, 10386, 18204, 28983, 41843, 100357, 123757, 141214, 156566, 192445, 215522, 222986,
    273675, 280051, 305883, 353177, 415231, 432191, 488471, 506665, 537639, 548464, 560671, 590826,
    609054, 629734, 644629, 672143, 680970, 735201, 759657, 773123,
)


def boundary_distance(fluid, P, T, z, out, salinity=None):
    """|TPD| distance of each converged answer from a phase boundary
    (oracle.ref.boundary_distance: non-trivial stability trials of the missing
    phases, zero for a present phase below a fraction of 1e-8)."""
    return ref.boundary_distance(fluid, P, T, z, out, salinity)


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
    P, T, z = synth.flash_points(1024, seed=104)
    make("flash_cpa_nc3.npz", make_cpa_h2o_co2_nc10(), P, T, z)
    labels_pr = lambda P, T, z, s, f=pr: ref.flash_batch(f, P, T, z, salinity=s, threads=8)["presence"]
    P, T, z = synth.boundary_points(512, labels_pr, seed=105)
    make("flash_boundary_pr_nc3.npz", pr, P, T, z)
    labels = lambda P, T, z, s, f=sw: ref.flash_batch(f, P, T, z, salinity=s, threads=8)["presence"]
    P, T, z, s = synth.boundary_points(256, labels, seed=106, salinity=True)
    make("flash_boundary_sw_nc3.npz", sw, P, T, z, s)
    nb = int(round(synth.BOUNDARY_FRACTION * (1 << 20)))
    P, T, z = synth.boundary_points(nb, labels_pr, seed=7919)
    np.savez_compressed(os.path.join(HERE, "bench_boundary_pr_nc3.npz"), P=P, T=T, z=z)
    P, T, z = synth.flash_points(1 << 20, seed=1)
    sel = np.array(RESCUED + FAILING)
    make("flash_continuation_pr_nc3.npz", pr, P[sel], T[sel], np.ascontiguousarray(z[:, sel]))


if __name__ == "__main__":
    main()
