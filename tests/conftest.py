import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA kernels)")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def ora():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def xg():
    import exageostat_b200 as xg
    from exageostat_b200 import build

    build.build()
    return xg


@pytest.fixture(scope="session")
def gpu(xg):
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    xg.init(0)
    return xg
