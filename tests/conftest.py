import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "online-physics-cuda_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU and the built libfe_b200.so")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests' device; they fail (not skip) when the library cannot reach one: no silent fallback."""
    import torch
    assert torch.cuda.is_available(), "the -m gpu tests need a GPU"
    from fieldcuda import _lib
    _lib.check(_lib.lib().fe_device_check())
    return torch.device("cuda:0")
