"""Shared pytest configuration.

``-m gpu`` selects the parity tests that run the CUDA library on a B200;
everything else (oracle vs golden vectors, host logic, library exports,
gloo multi-process tests) runs on the CPU.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def ccd_golden():
    return dict(np.load(os.path.join(GOLDEN, "ccd_golden.npz")))


@pytest.fixture(scope="session")
def ppe_golden():
    return dict(np.load(os.path.join(GOLDEN, "ppe_golden.npz")))


def golden_cases(golden, suffix):
    return sorted({k.split("/")[0] for k in golden if k.endswith(suffix)})


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch.device("cuda:0")
