"""pytest configuration: the `gpu` marker and shared fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def port():
    from oracle import pyoracle
    return pyoracle.Oracle("port")


@pytest.fixture(scope="session")
def ref():
    """The reference's own solver headers; skipped where they were not built."""
    from oracle import pyoracle
    if not os.path.exists(pyoracle.REF_LIB):
        try:
            pyoracle.build()
        except Exception:
            pass
    if not os.path.exists(pyoracle.REF_LIB):
        pytest.skip("reference build (oracle/_ref) not available")
    return pyoracle.Oracle("reference")
