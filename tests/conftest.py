import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "oneesan-gpu_b200")
for p in (PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libfdp.so")
    config.addinivalue_line("markers", "slow: longer-running CPU test")


@pytest.fixture(scope="session")
def engine():
    import fdp
    eng = fdp.Engine(0)
    yield eng
    eng.close()
