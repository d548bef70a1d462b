import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def read_env(p):
    env = {}
    for line in open(p):
        line = line.strip()
        if line and not line.startswith("#") and "=" in line:
            k, v = line.split("=", 1)
            env[k] = v
    return env


@pytest.fixture(scope="session")
def sample():
    import oracle as O
    n, idx, adj = O.read_egr(os.path.join(GOLDEN, "sample.egr"))
    env = read_env(os.path.join(GOLDEN, "sample.env"))
    return n, idx, adj, env


@pytest.fixture(scope="session")
def rmat12():
    import oracle as O
    return O.rmat_graph(12, 16, 1)


@pytest.fixture(scope="session")
def rmat16():
    import oracle as O
    return O.rmat_graph(16, 16, 1)
