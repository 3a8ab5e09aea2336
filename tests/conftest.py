"""Shared pytest set-up: markers, import paths and device fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "multigpu-vector_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ctx():
    """One mgv context on cuda:0 for the GPU tests."""
    import torch
    import mgv

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    torch.cuda.init()
    c = mgv.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    return torch
