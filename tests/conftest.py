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


def hand_graph(name):
    """Small hand graphs (undirected, unit weights, both directions listed):
    two K4 joined by one edge, a ring of 8 K5 (neighbouring cliques joined by
    one edge), a star on 10 vertices and a path on 12."""
    import itertools
    if name == "k4k4":
        e = list(itertools.combinations(range(4), 2)) + list(itertools.combinations(range(4, 8), 2)) + [(3, 4)]
        n = 8
    elif name == "ring_k5":
        e = []
        for c in range(8):
            b = 5 * c
            e += list(itertools.combinations(range(b, b + 5), 2))
            e.append((b + 4, (b + 5) % 40))
        n = 40
    elif name == "star":
        e, n = [(0, i) for i in range(1, 10)], 10
    elif name == "path":
        e, n = [(i, i + 1) for i in range(11)], 12
    else:
        raise ValueError(name)
    s, d, w = undirected_to_lists(e)
    return n, s, d, w
