import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    import __graft_entry__ as g
    return g.load_package()


@pytest.fixture(scope="session")
def wl():
    import __graft_entry__ as g
    return g.load_workload()


@pytest.fixture(scope="session")
def sys1(wl):
    return wl.make_system(1, (24, 24, 24))


@pytest.fixture(scope="session")
def sys2(wl):
    return wl.make_system(2, (48, 48, 48))


def rel_l2(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
