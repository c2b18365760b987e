"""Test configuration: the `gpu` marker, import paths, and in-tree builds.

Tests marked `gpu` need a CUDA device (a B200); everything else runs on CPU.
The checker libraries (oracle/) and the product library are built in place
with make when missing or stale, so a fresh checkout can run the suite.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cfd-simulator_b200")
for path in (ROOT, PKG, os.path.join(ROOT, "tests")):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    for target in (os.path.join(ROOT, "oracle"), PKG):
        subprocess.run(["make", "-s", "-C", target], check=True)
    # the reference-side binding's driver (a message only where the reference is absent)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "shim"], check=True)


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
