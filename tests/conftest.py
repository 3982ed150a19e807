import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running parity run")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build (if out of date) the CUDA library and the CPU oracle once per session."""
    from scale_b200 import build

    build.build_oracle()
    if not os.environ.get("SCALE_HEVI_SKIP_CUDA_BUILD"):
        build.build_cuda()
    yield


@pytest.fixture
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
