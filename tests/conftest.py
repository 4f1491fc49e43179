import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def kats():
    with open(os.path.join(HERE, "golden", "kats.json")) as f:
        return json.load(f)


def fnum(v):
    """JSON number or the strings 'nan' / 'inf' / '-inf'."""
    return float(v)
