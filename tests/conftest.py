import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu_lib():
    """The built library; GPU tests fail (not skip) when it cannot be built."""
    from asohf_b200 import build
    build.build()
    from asohf_b200 import api
    return api.load()


@pytest.fixture(scope="session")
def ctx(gpu_lib):
    from asohf_b200 import api
    a = api.Asohf(0)
    yield a
    a.close()
