import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.pyoracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def engine():
    """The CUDA engine on device 0. On a GPU host a failure here is a test failure, not a skip."""
    from sirius_b200.engine import Engine
    eng = Engine(0)
    yield eng
    eng.close()


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
