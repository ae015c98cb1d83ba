import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libmlbvh_b200.so")
    config.addinivalue_line("markers", "slow: full-size workloads (seconds of oracle time)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    import minimumlbvh_b200 as mb
    mb.lib()  # fails loudly when the library is missing
    return torch.device("cuda", 0)
