import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def orc():
    import oracle_py
    oracle_py.oracle()
    return oracle_py


@pytest.fixture(scope="session")
def engine():
    from gpudbmetalbenchmark_b200 import Engine
    e = Engine(0)
    yield e
    e.close()
