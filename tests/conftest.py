import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    if not os.path.exists(pyoracle.LIB_PATH):
        pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def capi():
    from multigpuegtsmoothing_b200 import capi as C
    C.lib()
    return C
