"""Test configuration: the `gpu` marker, import paths and shared helpers.

CPU tests (-m "not gpu") cover the oracle, the host logic and the C ABI
surface; GPU tests (-m gpu) are the parity tests proper and call the CUDA
path through the C ABI.
"""
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
PKG = REPO / "openstc-dev_b200"
for p in (str(PKG), str(REPO / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libostc.so")


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
