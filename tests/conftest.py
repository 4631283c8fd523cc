import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def schedules():
    with open(os.path.join(GOLDEN, "schedules.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_states():
    with np.load(os.path.join(GOLDEN, "states.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def native_lib():
    from frontierlabproject_b200 import _native
    from frontierlabproject_b200 import build
    build.build()
    return _native.lib()
