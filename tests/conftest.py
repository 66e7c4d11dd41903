"""Shared pytest configuration.

Markers:
  gpu — needs a CUDA device (B200); runs the CUDA path through the C ABI.
Everything unmarked runs on the CPU: the oracle against the reference's
golden fixtures, host-side logic, and the C-ABI library's exports.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device; exercises the CUDA path through the C ABI")


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_cuda():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this process")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
