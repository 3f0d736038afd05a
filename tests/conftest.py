import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for GPU tests; fails (never skips) without one, so a GPU
    run cannot pass by silently not running the kernels."""
    import torch

    assert torch.cuda.is_available(), "GPU test selected but no CUDA device is visible"
    import velodb_b200

    velodb_b200.lib()  # raises if the library was not built
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.lib()
    return oracle
