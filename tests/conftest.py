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


@pytest.fixture(autouse=True)
def _streaming_fault_flag(request):
    """After every GPU test: the streaming kernels' device fault flag (a bounded wait between warps
    that ran out) must be clear."""
    yield
    if request.node.get_closest_marker("gpu") is None:
        return
    try:
        import torch
        if not torch.cuda.is_available() or not torch.cuda.is_initialized():
            return
        from voxel_b200 import _lib
    except Exception:
        return
    assert _lib.device_status(clear=True) == 0, "a streaming operator kernel's bounded wait ran out"
