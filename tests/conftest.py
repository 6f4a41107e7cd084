import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "mumblebee.jl_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Bring the oracle (checker) and the product library up to date once per session: both builds
    compare source and object times, so an up-to-date tree costs only the checks, and a library
    older than its sources is rebuilt rather than tested as it is."""
    import oracle
    oracle.build()
    from build import build
    build()
    yield
