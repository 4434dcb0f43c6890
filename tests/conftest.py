"""Shared test set-up: import paths, the gpu marker, and parity helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("phase-field-project-3d_b200", "oracle", os.path.join("tests", "golden")):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running parity case")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return True


# FP64 parity bound of the plain form against the CPU oracle: max |a-b| over
# the field <= RTOL * max|b| (CUDA's and glibc's log may differ by 1 ulp, so
# the fields are not bit-identical; everything else is).
RTOL_FP64 = 1e-12


def max_rel(a: np.ndarray, b: np.ndarray) -> float:
    scale = float(np.max(np.abs(b)))
    if scale == 0.0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b))) / scale
