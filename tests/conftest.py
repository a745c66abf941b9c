"""Shared fixtures: build the CPU oracle once; register the gpu marker."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libffs_lbm.so")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    yield


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from freeflow_b200 import load
    load()  # fails loudly if the product library is missing
    return torch.device("cuda:0")
