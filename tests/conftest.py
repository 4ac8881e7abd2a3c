import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the libpmg_b200 kernels")


@pytest.fixture(scope="session")
def pmg():
    """The product package; GPU tests fail (not skip) when no device is present."""
    import parmoon_b200 as P
    import ctypes
    n = ctypes.c_int(0)
    rc = P.lib().pmg_device_count(ctypes.byref(n))
    if rc != 0 or n.value < 1:
        pytest.fail("no CUDA device visible to libpmg_b200")
    return P


@pytest.fixture(scope="session")
def oracle():
    from oracle import cd3d
    cd3d.build()
    return cd3d


def golden(name):
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
