import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: longer CPU reference runs")


@pytest.fixture(scope="session", autouse=True)
def _build_libraries():
    """Build the oracle and libamdk once per session (nvcc cross-compiles)."""
    from oracle import oracle as orc
    orc.build()
    from amdkiit_b200 import build
    build.build()
