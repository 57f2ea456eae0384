import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def built_lib():
    """libpgmpm.so built in-tree (nvcc cross-compiles without a GPU)."""
    from physgrad_b200 import build

    return build.build()


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle

    if not os.path.exists(pyoracle.LIB_PATH):
        pyoracle.build(with_ref=False)
    return pyoracle


@pytest.fixture(scope="session")
def gpu(built_lib):
    if not _cuda_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    import physgrad_b200

    physgrad_b200.lib()
    return physgrad_b200
