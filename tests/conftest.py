import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libcpstep.so")


@pytest.fixture(scope="session", autouse=True)
def _built_library():
    """Build libcpstep.so in-tree when it is missing or stale (nvcc, no GPU needed)."""
    from openatom_b200 import build as b
    if not b.up_to_date():
        if not os.path.exists(b.NVCC):
            pytest.exit("libcpstep.so is not built and nvcc is unavailable", 2)
        b.build()
    yield


def ref_lib():
    """oracle/_ref/libref.so (reference leaves compiled from source) or None."""
    import ctypes
    p = os.path.join(ROOT, "oracle", "_ref", "libref.so")
    if not os.path.exists(p):
        return None
    return ctypes.CDLL(p)


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
