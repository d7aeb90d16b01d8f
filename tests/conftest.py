import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


def plummer(n, seed=0, b=1.0, size=-1.0):
    from hierarquicos_b200.initial_values import generate_initial_values

    m, q, _ = generate_initial_values(n, size, -1.0, True, False, "plummer", (1.0, b), seed=seed,
                                      velocities=False)
    return m, q


def hernquist(n, seed=0, a=1.0, size=100.0):
    from hierarquicos_b200.initial_values import generate_initial_values

    m, q, _ = generate_initial_values(n, size, -1.0, True, False, "hernquist", (1.0, a), seed=seed,
                                      velocities=False)
    return m, q


def xyz(q):
    return (np.ascontiguousarray(q[:, 0]), np.ascontiguousarray(q[:, 1]),
            np.ascontiguousarray(q[:, 2]))
