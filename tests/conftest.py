"""Shared pytest configuration.

Tests marked `gpu` need a CUDA device and libdiffsoup_b200.so; everything else
runs on CPU (oracle against the golden fixtures, host logic, ABI exports).
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["config1_small", "config2_small", "edge_cases"]


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    return {name: dict(np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))) for name in GOLDEN_CASES}
