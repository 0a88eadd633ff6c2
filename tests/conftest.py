import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def ref_available() -> bool:
    from oracle.oracle import ref_library
    return ref_library() is not None


@pytest.fixture(scope="session")
def lib():
    from alebgk4paper_b200 import build, _abi
    build.build()
    return _abi.load()


@pytest.fixture(scope="session")
def gpu():
    """Skips unless a CUDA device is visible; the library must then load."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from alebgk4paper_b200 import _abi
    return _abi.load()
