import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not _cuda_available():
        pytest.skip("no CUDA device")
    import torch
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def qcu_lib():
    """The product library; built in-tree if it is missing (nvcc cross-compiles)."""
    import qcu_cg_inverter_b200 as q
    if not os.path.exists(q.LIB_PATH):
        q.build_library()
    return q


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O
