import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (run with -m gpu)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def rtwlib():
    """The product library (built if missing: nvcc cross-compiles without a GPU)."""
    from rtwca_b200 import abi, build
    if not abi.LIB_PATH.exists():
        build.build()
    return abi.load()


@pytest.fixture(scope="session")
def renderer(rtwlib):
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    from rtwca_b200 import Renderer
    r = Renderer(0)
    yield r
    r.close()
