import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the libcfd2lcs_b200 device path")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_dp():
    from oracle.oracle import Oracle
    return Oracle("dp")


@pytest.fixture(scope="session")
def oracle_sp():
    from oracle.oracle import Oracle
    return Oracle("sp")
