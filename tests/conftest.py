"""Shared test set-up: import paths, the gpu marker, the built libraries."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "numi-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _make(path):
    subprocess.run(["make", "-s", "-C", path], check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the product library and the oracle once per session."""
    _make(os.path.join(ROOT, "numi-solver_b200"))
    _make(os.path.join(ROOT, "oracle"))


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
