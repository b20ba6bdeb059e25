"""Shared test setup: import paths, the `gpu` marker and golden fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "qbox-public_b200")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"ref_{name}.npz")))


@pytest.fixture
def load_golden():
    return golden
