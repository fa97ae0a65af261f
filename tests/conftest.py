"""Shared test configuration: the `gpu` marker, repository paths and golden-fixture loaders."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


def golden(name):
    path = GOLDEN / name
    if path.suffix == ".json":
        return json.loads(path.read_text())
    with np.load(path) as f:
        return {k: f[k] for k in f.files}


@pytest.fixture(scope="session")
def gold():
    return golden
