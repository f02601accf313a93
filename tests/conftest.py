"""Shared test configuration.

``-m gpu`` tests need a CUDA device (B200) and exercise the product path
through the C ABI; every other test runs on the CPU.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (str(ROOT), str(GOLDEN)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100a) device; run with -m gpu")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device; GPU tests fail (not skip) when there is none."""
    import torch

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    import shearwave_b200._native as native

    native.load()
    return torch.device("cuda", 0)
