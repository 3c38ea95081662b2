import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libpa_b200.so")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import build
    build.build()
    from oracle import cpu
    return cpu


@pytest.fixture(scope="session")
def pa():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import platoanalyze_b200
    return platoanalyze_b200
