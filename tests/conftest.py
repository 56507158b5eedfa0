import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    out = {}
    d = os.path.join(ROOT, "tests", "golden")
    for f in sorted(os.listdir(d)):
        if f.endswith(".npz"):
            out[f[:-4]] = dict(np.load(os.path.join(d, f)))
    return out
