import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the device path")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lpm():
    return importlib.import_module("lpm-cpp_b200.lpm")


@pytest.fixture(scope="session")
def cfg():
    return importlib.import_module("lpm-cpp_b200.configs")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    return O
