import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "rvs-cuda_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    # GPU tests fail loudly rather than skip when the device is missing, but
    # only when they were selected explicitly (-m gpu).
    pass


@pytest.fixture(scope="session")
def ctx():
    import rvsb
    c = rvsb.Context(0)
    yield c
    c.close()
