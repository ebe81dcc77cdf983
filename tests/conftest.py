import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs the CUDA path")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build libultraprecise.so and the CPU oracle when they are missing."""
    from ultraprecise_b200 import abi
    if not os.path.exists(abi.LIB_PATH):
        from ultraprecise_b200 import build
        build.build()
    from oracle import oracle
    oracle.load()
    yield


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
