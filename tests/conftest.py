import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference's one shipped graph (SNAP wiki-Vote, bundled at the root of
# sixt99/TriBIT): a copy is committed beside the other golden fixtures;
# TRIBIT_WIKI_VOTE points the tests at another copy.
WIKI_VOTE = os.environ.get("TRIBIT_WIKI_VOTE", os.path.join(ROOT, "tests", "golden", "wiki-Vote.mtx"))
WIKI_VOTE_SHA256_16 = "c28b16ffed623c7f"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def counter():
    import tribit_b200 as tb
    c = tb.Counter()
    yield c
    c.close()
