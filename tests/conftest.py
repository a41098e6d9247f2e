import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libscattersim_b200.so")


@pytest.fixture(scope="session")
def ctx():
    from scattersim_b200.solver import Context
    c = Context(0)
    yield c
    c.close()
