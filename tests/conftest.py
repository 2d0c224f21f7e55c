import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def engine():
    import clwilson_b200 as wl
    e = wl.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="session")
def golden():
    import json
    d = os.path.join(ROOT, "tests", "golden")
    out = {}
    for name in ("kat", "small", "range_1e5", "capped", "nonresidue"):
        with open(os.path.join(d, name + ".json")) as f:
            out[name] = json.load(f)
    return out
