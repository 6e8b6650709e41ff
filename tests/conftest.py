import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the native library and the oracle (no-ops when up to date)."""
    from subgraph_b200 import build as b
    from oracle import oracle as O
    b.build()
    O.build()
    yield


@pytest.fixture(scope="session")
def golden():
    from tests.helpers import Golden
    return Golden()
