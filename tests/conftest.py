import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def species():
    from combustioncodegpu_b200 import cases
    return cases.synthetic_species()


@pytest.fixture(scope="session")
def cclib():
    """The product library, built in-tree for sm_100a."""
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import build
    build.build()
    return cc.load_library()


def has_gpu():
    try:
        import combustioncodegpu_b200 as cc
        return cc.device_count() > 0
    except Exception:
        return False
