import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pgfem-3d_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build (if stale) the product library and the oracle before any test."""
    import build as pkg_build  # pgfem-3d_b200/build.py
    pkg_build.build()
    import oracle
    oracle.build()
    yield


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.fail("GPU test needs a CUDA device")
    import torch
    torch.cuda.init()
    return torch.device("cuda:0")
