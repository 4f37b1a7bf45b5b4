import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU oracle check")


@pytest.fixture(scope="session")
def cuda_device():
    """Skips only when the machine has no CUDA device; the library itself
    must be present (a missing library fails the test)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from uq_b200 import native

    native.lib()
    return 0
