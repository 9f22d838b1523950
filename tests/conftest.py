"""Shared test configuration: the ``gpu`` marker and golden-fixture helpers."""

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def known_answers():
    return json.loads((GOLDEN / "known_answers.json").read_text())


def cols(pairs):
    a = np.asarray(pairs, dtype=np.uint32).reshape(-1, 2)
    return a[:, 0].copy(), a[:, 1].copy()


def pairs(columns):
    return [[int(a), int(b)] for a, b in zip(*columns)]


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test without a CUDA device")
    from sparkalog_b200 import _native

    _native.load()
    return torch
