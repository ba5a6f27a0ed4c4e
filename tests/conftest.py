import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library through its C ABI")


def load_golden(name):
    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        meta = json.load(f)
    path = os.path.join(GOLDEN, f"{name}.npz")
    arrays = dict(np.load(path)) if os.path.exists(path) else {}
    return meta, arrays


@pytest.fixture(scope="session")
def golden():
    return load_golden
