import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def orc():
    from oracle import pyorc
    pyorc.load()
    return pyorc


@pytest.fixture(scope="session")
def golden_qmc():
    import numpy as np
    return np.load(os.path.join(GOLDEN, "qmc_golden.npz"))


@pytest.fixture(scope="session")
def golden_rates():
    import numpy as np
    return np.load(os.path.join(GOLDEN, "rates_golden.npz"))
