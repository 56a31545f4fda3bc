import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the library's kernels")


@pytest.fixture
def no_cuda_device():
    """For host-logic tests that hand the library placeholder device addresses
    which the call under test must reject before any device work.  They run
    only where no CUDA device is visible, so that a changed check order can
    never launch a kernel on those addresses."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("placeholder device addresses: runs only where no CUDA device is visible")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    torch.cuda.init()
    return torch.device("cuda:0")
