"""Shared pytest configuration.

``gpu``-marked tests need a CUDA device and the in-tree extension; the CPU
suite (``-m "not gpu"``) covers the oracle against the golden fixtures, the
host-side logic and the C-ABI library's exported symbols.
"""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built extension")


@pytest.fixture
def golden():
    import numpy as np

    def load(name):
        return np.load(GOLDEN / name)

    return load
