import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu():
    """Skips nothing: a gpu-marked test on a box without a GPU must fail loudly."""
    import torch  # noqa: F401  (plumbing only: device presence)
    assert torch.cuda.is_available(), "gpu test run without a CUDA device"
    return 0
