import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built libbespoke_gpu.so")


@pytest.fixture(scope="session")
def engine():
    from bespokeolap_artifacts_b200.engine import Engine

    e = Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="session")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch
