import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through the C ABI")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the native libraries once (no-op when they are up to date)."""
    from lda_sc20_b200 import build
    build.build_all()
    yield
