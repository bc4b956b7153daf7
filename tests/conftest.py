import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# Load the engine library (and with it the toolkit's cuSOLVER / cuBLAS) before any test module imports torch,
# whose bundled copies would otherwise be shared by soname.
try:
    from xatu_b200 import _lib as _engine_lib
    if os.path.exists(_engine_lib.LIB_PATH):
        _engine_lib.lib()
except OSError:
    pass


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: larger sizes")


@pytest.fixture(scope="session", autouse=True)
def _build_native():
    """Build the oracle's C part and (if nvcc exists) the engine library once per session."""
    from oracle import build as ob
    ob.build()
    try:
        from xatu_b200 import build as xb
        xb.build()
    except RuntimeError:
        pass
    yield
