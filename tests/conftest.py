import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def ocip():
    """The ctypes mirror of the C ABI (fails loudly if the library is missing)."""
    from openclipp_b200 import ocip as mod
    return mod


@pytest.fixture(scope="session")
def ctx(ocip):
    """One GPU context for the whole session (PLAIN path unless a test sets another)."""
    c = ocip.Context()
    yield c
    c.close()


@pytest.fixture
def plain(ctx, ocip):
    ctx.make_current()
    ctx.set_path(ocip.PATH_PLAIN)
    yield ctx
    ctx.set_path(ocip.PATH_PLAIN)


@pytest.fixture
def tensor(ctx, ocip):
    ctx.make_current()
    ctx.set_path(ocip.PATH_TENSOR)
    yield ctx
    ctx.set_path(ocip.PATH_PLAIN)
