import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def tan_ctx():
    """One TANContext on cuda:0 for the GPU tests (fails loudly without the library)."""
    from tan_b200 import TANContext

    ctx = TANContext(0)
    yield ctx
    ctx.Release()
