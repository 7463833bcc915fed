"""Shared pytest configuration: the ``gpu`` marker and golden-fixture access."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name):
    """Load one committed golden fixture (``.npz``/``.npy``/``.json``)."""
    path = os.path.join(GOLDEN, name)
    if name.endswith(".json"):
        import json

        with open(path) as fh:
            return json.load(fh)
    return np.load(path)


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = float(np.linalg.norm(b.ravel()))
    num = float(np.linalg.norm((a - b).ravel()))
    return num / den if den else num


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    return torch.device("cuda:0")
