import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
PACKAGE = "jax-pytorch-vlasov_b200"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def load_package():
    """The package directory name is not a Python identifier, so it is
    imported through importlib."""
    return importlib.import_module(PACKAGE)


@pytest.fixture(scope="session")
def vp():
    return load_package()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
        return cache[name]

    return get
