import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU; run with -m gpu")


@pytest.fixture(scope="session")
def built_lib():
    """Builds librls_b200.so if its sources are newer (nvcc cross-compiles without a GPU)."""
    from rls_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def cuda_device(built_lib):
    """The GPU tests require a device: they fail (never skip) without one."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device visible: GPU tests need a B200")
    return 0
