import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "raptor_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


def golden_csr(g, name):
    m, n = (int(v) for v in g[name + "__shape"])
    return m, n, g[name + "__rowptr"], g[name + "__cols"], g[name + "__vals"]
