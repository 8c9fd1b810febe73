import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def relerr(got, ref, floor=0.0):
    """Norm-wise relative error max|got-ref| / max(max|ref|, floor)."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    scale = max(float(np.abs(ref).max()) if ref.size else 0.0, floor)
    if scale == 0.0:
        return float(np.abs(got - ref).max()) if ref.size else 0.0
    return float(np.abs(got - ref).max()) / scale


@pytest.fixture(scope="session")
def gpu():
    from mpm_b200 import _abi
    _abi.load()
    n = _abi.device_count()
    assert n >= 1, "GPU tests need a CUDA device"
    return n
