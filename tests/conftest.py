import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and the built libscgpu.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    O.use_reference_fft(False)
    return O


@pytest.fixture(scope="session")
def gpu():
    """The C-ABI binding; GPU tests fail loudly (no skip) when the device or
    the library is missing."""
    import torch

    assert torch.cuda.is_available(), "GPU test selected but no CUDA device is visible"
    from src_b200 import scgpu
    scgpu.lib()
    return scgpu
