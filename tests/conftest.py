"""Shared pytest configuration: the ``gpu`` marker and fixture helpers."""

from __future__ import annotations

import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a B200)")


def load_golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as data:
        return {key: data[key] for key in data.files}


def golden_mvp_names() -> list:
    names = []
    for path in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        name = os.path.splitext(os.path.basename(path))[0]
        if name not in ("canonical_known_answers", "integral_known_answer"):
            names.append(name)
    return names
