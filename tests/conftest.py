import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the native library")
    config.addinivalue_line("markers", "slow: long-running full-size case")


@pytest.fixture(scope="session", autouse=True)
def _native_built():
    """Build the native library and the oracle in-tree when sources are newer (nvcc cross-compiles)."""
    from sqsgenerator_b200 import build as native_build
    from oracle import build as oracle_build

    native_build.build()
    oracle_build.build()
