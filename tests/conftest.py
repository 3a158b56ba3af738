import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: full-size workload, minutes on CPU")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name), allow_pickle=False)

    return load


@pytest.fixture(scope="session")
def matrix_txt(golden):
    """cuda_test/matrix.txt of the reference as (rowptr, col, signed values, m, n)."""
    z = golden("matrix_txt.npz")
    return z["rowptr"], z["col"], z["val"], int(z["m"]), int(z["n"])


@pytest.fixture(scope="session")
def ctx():
    import rust_rank_b200 as rr

    return rr.Context(0)
