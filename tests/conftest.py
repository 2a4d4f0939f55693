import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) CUDA device")


@pytest.fixture(scope="session")
def dev():
    """The CUDA device for GPU tests.  No skip: a GPU test that runs without a
    device must fail, so a missing GPU or library is never a silent pass."""
    import torch
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from opensycl_b200 import capi
    capi.lib()
    return torch.device("cuda:0")
