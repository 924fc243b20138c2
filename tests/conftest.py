import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built libbp_b200.so")
    config.addinivalue_line("markers", "slow: full-size cases (minutes)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def bp():
    import benchparanumal_b200 as B
    B.lib()
    return B


@pytest.fixture(scope="session")
def gpu(bp):
    """The product library with device 0 initialised (GPU tests only)."""
    bp.platform_init(0)
    return bp
