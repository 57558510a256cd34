import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import ix_oracle

    ix_oracle.build()
    return ix_oracle


@pytest.fixture(scope="session")
def backend():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from indicatrix_b200.backend import GpuBackend

    b = GpuBackend.acquire()
    assert b.available, "libix_cuda.so loaded but no backend could be created"
    yield b
    b.close()


@pytest.fixture(scope="session")
def exact_backend():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from indicatrix_b200 import abi
    from indicatrix_b200.backend import GpuBackend

    b = GpuBackend.acquire(precision=abi.PRECISION_EXACT)
    assert b.available
    yield b
    b.close()
