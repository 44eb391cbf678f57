import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REFERENCE_WIKI_VOTE = "/root/reference/wiki-Vote.mtx"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def counter():
    import tribit_b200 as tb
    c = tb.Counter()
    yield c
    c.close()
