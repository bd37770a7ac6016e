import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the solver through the C ABI")


@pytest.fixture(scope="session")
def steps_lib():
    """The in-tree libsteps_b200.so (built if missing or stale)."""
    from steps_b200 import _lib, build

    build.build()
    return _lib.load()
