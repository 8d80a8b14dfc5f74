import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs an sm_100 GPU and the built libsparc_gpu.so")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    import oracle
    oracle.build()
    yield
