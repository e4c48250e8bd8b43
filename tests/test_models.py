"""CPU checks of the multi-model workload and of the nz_model_io record."""
import ctypes as C

import numpy as np

from nonenone_b200 import abi, synth


def test_model_batch_specs_shape_and_determinism():
    a = synth.model_batch_specs(256, seed=5)
    b = synth.model_batch_specs(256, seed=5)
    assert a == b
    ncs = {nc for nc, _, _ in a}
    assert ncs == set(synth.MODEL_NCS)
    assert {e for _, e, _ in a} == set(synth.MODEL_EOS)
    sizes = np.array([n for _, _, n in a])
    assert sizes.min() >= 1.0e4 - 1 and sizes.max() <= 5.0e5
    # log-uniform: the median is near the geometric mean of the bounds
    assert 3.0e4 < np.median(sizes) < 1.5e5
    w = synth.model_batch_specs(2000, seed=6, eos_weights=[0.5, 0.3, 0.2])
    frac = np.mean([e == "pr" for _, e, _ in w])
    assert abs(frac - 0.5) < 0.05


def test_model_points_follow_the_hydrostatic_case():
    P, T, z, sal = synth.model_points(6, 5000, seed=3)
    depth = (P - 20.0e6) / 0.01e6
    assert depth.min() >= 0.0 and depth.max() <= 250.0
    assert np.allclose(T, 373.15 + 0.03 * depth)
    assert z.shape == (6, 5000) and np.allclose(z.sum(axis=0), 1.0)
    # Dirichlet(4, 2, 1, 1, 1, 1): mean fractions 0.4, 0.2, 0.1, ...
    assert np.allclose(z.mean(axis=1), [0.4, 0.2, 0.1, 0.1, 0.1, 0.1], atol=0.01)
    assert sal.min() >= 0.0 and sal.max() <= 2.0


def test_model_io_record_layout():
    # four input pointers, then the ten nz_flash_out pointers
    assert C.sizeof(abi.ModelIO) == 14 * C.sizeof(C.c_void_p)
    assert abi.ModelIO.out.offset == 4 * C.sizeof(C.c_void_p)
