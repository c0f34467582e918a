"""Shared pytest setup: package path, the `gpu` marker, skip rules.

Tests marked `gpu` need a CUDA device and the built lib/libitr_gpu.so; everything else
runs on the CPU (oracle checks against the reference's published values, host logic,
C-ABI symbol exports, multi-process gloo tests).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "inverse-terrain-engine_b200")
for p in (PKG, os.path.join(ROOT, "tests"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (CUDA) and the built CUDA library")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
