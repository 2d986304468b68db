import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Build the CUDA library and the oracle once per session (no GPU needed)."""
    from oracle.build import build_oracle
    from szsnn_b200.build import build

    build()
    build_oracle()
    return True


@pytest.fixture(scope="session")
def ctx(built):
    import szsnn_b200 as sz

    c = sz.Context(0)
    yield c
    c.close()
