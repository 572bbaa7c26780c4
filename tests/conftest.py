import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def basics():
    with open(os.path.join(GOLDEN, "test_basics_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ref_cases():
    with open(os.path.join(GOLDEN, "ref_cases.json")) as f:
        return json.load(f)
