"""Shared pytest configuration.

Markers: ``gpu`` (needs a CUDA device and liblbm_b200.so; these are the parity
tests proper) and ``slow``. On a machine without CUDA the ``gpu`` tests are
skipped; on a machine with CUDA they run and fail loudly if the library is
missing -- there is no fallback path to hide behind.
"""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import lbm_b200  # noqa: E402,F401  (registers the package under its import name)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built liblbm_b200.so")
    config.addinivalue_line("markers", "slow: long runs")


def _cuda_present() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except ImportError:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_present():
        return
    skip = pytest.mark.skip(reason="no CUDA device on this machine")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
