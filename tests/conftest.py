import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)  # test helpers (textio_cases)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def native_lib():
    """The library under test; built if it is missing (nvcc cross-compiles)."""
    from hpgl_b200 import build, native
    if not os.path.exists(native.LIB_PATH):
        build.build()
    return native.lib()
