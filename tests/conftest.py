import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def ykb_lib():
    """libykb.so, built in-tree if missing (nvcc cross-compiles without a GPU)."""
    from fdk_cuda_impl_b200 import build as B
    B.build()
    from fdk_cuda_impl_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def cuda_device(ykb_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("CUDA device unavailable")
    torch.cuda.init()
    return 0
