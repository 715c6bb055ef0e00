import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "ceos-eems_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "hexa8_svk.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_nh():
    with open(os.path.join(ROOT, "tests", "golden", "hexa8_nh_q1p0.json")) as f:
        return json.load(f)
