import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "lua-santoku-tsetlin_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def tm():
    """The product package; GPU tests need it built and a device present."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    import santoku_tsetlin
    santoku_tsetlin.lib()
    return santoku_tsetlin
