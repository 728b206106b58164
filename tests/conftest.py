import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")
    config.addinivalue_line("markers", "slow: production-size case (minutes of oracle time)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def bph():
    import bipoly_hydro_b200 as B
    from bipoly_hydro_b200 import build as bb

    bb.build()
    return B
