import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs the CUDA path")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.set_threads(os.cpu_count() or 1)
    return oracle


@pytest.fixture(scope="session")
def box22():
    """The 22^3, p = 8 Taylor-Green box (built once per session for the tests that need it)."""
    from dsem_b200 import mesh
    return mesh.Box(22, 22, 22, 8)
