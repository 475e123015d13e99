import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libbastr_gpu.so")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def gpu_lib():
    """Builds (if stale) and loads the CUDA library; GPU tests fail loudly without it."""
    from bastr_b200 import build as _b
    _b.build()
    from bastr_b200 import load_library
    return load_library()
