import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_available():
    return _has_gpu()


@pytest.fixture(scope="session")
def product_lib():
    """The CUDA library; on a GPU host its absence is an error, never a fallback."""
    from ice_fem_2025a_b200 import abi, build
    if not os.path.exists(abi.product_library_path()):
        build.build()
    return abi.load_product()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as orc
    return orc.lib()
