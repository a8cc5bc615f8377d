import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the engine's kernels)")


@pytest.fixture(scope="session", autouse=True)
def native_build():
    """Build the engine, generator, driver and the oracle (incremental)."""
    from nise_2017_b200 import build
    import oracle
    build.build_all()
    oracle.build(ref=oracle.reference_present())
