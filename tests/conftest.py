import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def oracle():
    from oracle import dense

    dense.load()
    return dense


@pytest.fixture(scope="session")
def gpu():
    """The product library on a live device; fails loudly if either is missing."""
    import torch

    from algebra_linear_b200 import _lib

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    lib = _lib.load()
    torch.cuda.init()
    return lib
