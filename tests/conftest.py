import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libvship.so")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def vship_lib():
    from vship_b200 import build, api
    build.build()
    return api.load()


@pytest.fixture(scope="session")
def gpu(vship_lib):
    if not _has_gpu():
        pytest.fail("GPU test run without a visible CUDA device")
    return vship_lib
