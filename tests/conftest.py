import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built libgs3d_cuda.so")


@pytest.fixture(scope="session")
def ctx():
    """One gs3dc context for the GPU tests of the session."""
    from aaags_claude_b200 import gs3d
    c = gs3d.Context(0)
    yield c
    c.close()
