"""Shared pytest configuration.

Markers: `gpu` tests need a CUDA device and the built libnfx_b200.so; the rest
run on the CPU.  The oracle under oracle/ is the checker for every parity test.
"""

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture
def rng():
    return np.random.default_rng(42)


def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return torch.device("cuda", 0)


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))
