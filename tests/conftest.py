import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libsgr.so")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle (test infrastructure) if it is missing; the product library is built by
    __graft_entry__.build() and is never rebuilt implicitly by the GPU tests."""
    from oracle import oracle as O
    if not os.path.exists(O.LIB):
        O.build()
    yield
