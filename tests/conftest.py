"""Shared pytest configuration.

Marker ``gpu``: the test needs a CUDA device (run with ``-m gpu`` on a B200);
everything else runs on the CPU (``-m "not gpu"``).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("this test needs a CUDA device")
    from transportse_b200 import build
    build.build()
    return torch.device("cuda:0")
