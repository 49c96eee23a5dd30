import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session")
def dsss():
    """The package (libdsss over ctypes); builds the library if it is missing."""
    mod = __graft_entry__.load_package()
    if not os.path.exists(mod.LIB_PATH):
        __graft_entry__.build()
    mod.lib()
    return mod


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def ctx(dsss):
    c = dsss.Context(0)
    yield c
    c.close()
