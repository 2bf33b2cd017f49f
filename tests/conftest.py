import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product kernels")
    config.addinivalue_line("markers", "slow: large inputs (seconds of CPU work)")


@pytest.fixture(scope="session")
def cuda_device():
    """The GPU tests run the CUDA kernels; without a GPU they fail, never fall back."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu-marked test needs a CUDA device (there is no CPU fallback)")
    torch.cuda.init()
    return 0

