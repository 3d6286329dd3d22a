import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on a B200)")


@pytest.fixture(scope="session")
def ctx():
    import hyteg_b200 as H

    c = H.Context(0)
    yield c
    c.close()
