import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger sizes")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture(scope="session")
def fixtures():
    import numpy as np
    from oracle import OBJ_DTYPE
    a = np.fromfile(os.path.join(GOLDEN, "test.idradec"), OBJ_DTYPE)
    a2 = np.fromfile(os.path.join(GOLDEN, "test2.idradec"), OBJ_DTYPE)
    return a, a2


@pytest.fixture(scope="session")
def ctx():
    import xmatch_b200 as xm
    c = xm.Context(0)
    yield c
    c.close()
