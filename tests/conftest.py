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


def octree_leaf_list(path, boxlen, base_level=2, max_level=5, p_split=0.35, seed=7, n0=100.0):
    """A small irregular octree for the parity tests: every cell of levels
    base_level..max_level-1 splits with probability p_split (seeded), so face
    neighbours differ by up to max_level - base_level levels; n_H varies
    smoothly around n0.  Writes the text leaf list, returns the leaf count."""
    import numpy as np
    from mochii_b200 import amr
    rng = np.random.default_rng(seed)

    def refine(x, y, z, lev):
        r = np.sqrt(x * x + y * y + z * z) / boxlen
        return rng.random(np.shape(x)) < p_split * (1.5 - r)

    def dens(x, y, z, lev):
        return n0 * np.exp(0.4 * np.sin(6.0 * x / boxlen) * np.cos(5.0 * y / boxlen) + 0.2 * z / boxlen)

    x, y, z, lev, nH = amr.build_leaves(boxlen, base_level, max_level, refine, dens)
    amr.write_leaf_list(path, boxlen, x, y, z, lev, nH)
    return len(x)
