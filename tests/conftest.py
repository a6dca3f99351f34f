import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "pdot.jl_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) CUDA device")


@pytest.fixture(scope="session")
def built():
    """Build libpdot.so and the oracle once per session (no GPU needed)."""
    import __graft_entry__

    __graft_entry__.build()
    return True


@pytest.fixture(scope="session")
def cuda(built):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    torch.cuda.set_device(0)
    return torch.device("cuda", 0)
