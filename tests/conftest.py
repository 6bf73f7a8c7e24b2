"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and run the native library; all
others run on the CPU (oracle, host logic, library exports)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the native library")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/libmaosref.so is not built (make -C oracle ref)")
    return ref
