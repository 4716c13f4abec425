import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_package():
    """Import the product package (its directory name carries hyphens)."""
    return importlib.import_module("gpu-wm-next_b200")


@pytest.fixture(scope="session")
def gwm():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle
