import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    if not os.path.exists(O._LIB):
        O.build()
    return O


@pytest.fixture(scope="session")
def gen():
    from louvaingpu_b200 import graphgen
    return graphgen


def undirected_to_lists(und, weights=None):
    import numpy as np
    und = list(und)
    if weights is None:
        weights = [1.0] * len(und)
    src = [a for a, b in und] + [b for a, b in und]
    dst = [b for a, b in und] + [a for a, b in und]
    w = list(weights) + list(weights)
    return np.array(src, np.int32), np.array(dst, np.int32), np.array(w, np.float32)
