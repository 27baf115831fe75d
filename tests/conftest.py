import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "modem-gpu_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _cuda_available() -> bool:
    try:
        from mt3d import capi
        return capi.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not _cuda_available():
        pytest.fail("no CUDA device / libmt3d.so not loadable: the GPU tests need the CUDA library on a B200")
    return True
