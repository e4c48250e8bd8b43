import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        with np.load(os.path.join(GOLDEN, name)) as f:
            return {k: f[k] for k in f.files}
    return load


@pytest.fixture(scope="session")
def reference():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref (the compiled reference) is not built here")
    return ref
