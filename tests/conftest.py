"""Shared pytest configuration: the ``gpu`` marker and oracle availability."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def reference_lib():
    """The compiled reference CPU library (oracle/_ref), skipping when it is absent."""
    import oracle
    lib = oracle.reference()
    if lib is None:
        pytest.skip("reference CPU library (oracle/_ref/libzkx_ref.so) is not built")
    return lib
