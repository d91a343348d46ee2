"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Build libfwi2d.so and the oracle libraries in-tree if they are missing."""
    from fwi2d_b200 import build as b
    if not b.LIB.exists():
        b.build()
    from oracle import oracle as O
    for bits in (64, 32):
        if not (O.HERE / f"liboracle{bits}.so").exists():
            O.build()
    return True


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
