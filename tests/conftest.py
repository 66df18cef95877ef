import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def published():
    """The reference's published results for its force path (golden values,
    tests/golden/reference_published.json, written by make_published.py from
    the reference's own text files)."""
    import json

    with open(os.path.join(ROOT, "tests", "golden", "reference_published.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden():
    return published()


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.lib()
    return oracle
