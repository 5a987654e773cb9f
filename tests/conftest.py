import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def ctx():
    from experiments_b200 import b3
    c = b3.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def host_ctx():
    from experiments_b200 import b3
    c = b3.Context(-1)
    yield c
    c.close()
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)
