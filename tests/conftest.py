import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle and libnsegpu.so in-tree if they are missing."""
    from oracle import oracle as O
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        O.build()
    from vtkmakecompare_b200 import build as B
    if not os.path.exists(B.LIB):
        B.build()
    yield
