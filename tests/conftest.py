import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: a benchmark-size case (minutes)")


@pytest.fixture(scope="session")
def built():
    """Build the native libraries in-tree (no-op when up to date)."""
    from coincgraph_b200 import build

    build.build_all()
    import oracle.build as ob

    ob.build_oracle()
    ob.build_ref()
    return True
