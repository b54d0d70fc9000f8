import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def fk():
    """The product package with its library built."""
    import fteik_b200
    if not os.path.exists(fteik_b200.LIB_PATH):
        fteik_b200.build()
    fteik_b200.lib()
    return fteik_b200
