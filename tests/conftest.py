import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Build (if stale) the CUDA libraries and the oracle."""
    from emsolver_b200 import build as B
    from oracle import build_oracle
    B.build()
    build_oracle()
    return True


def golden(name):
    import numpy as np
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.fail(f"golden fixture {path} is missing (tests/golden/make_golden.py)")
    return dict(np.load(path, allow_pickle=False))
