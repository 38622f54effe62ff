import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on a B200)")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def wt():
    import wtet_b200
    import wtet_b200.build as b

    b.build()
    wtet_b200._core.load()
    return wtet_b200


@pytest.fixture(scope="session")
def gpu(wt):
    if not cuda_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    return wt
