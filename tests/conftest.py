"""Shared test configuration.

Markers: `gpu` -- needs a CUDA device (the parity tests proper, run on a
B200); everything else runs on CPU.  The CPU oracle (oracle/) is the
checker and is built on demand.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import build, pyoracle
    build.build()
    return pyoracle


@pytest.fixture(scope="session")
def engine_lib():
    """The product library, built in-tree (fails loudly if it cannot be)."""
    from smaug_b200 import build, engine
    build.build()
    return engine
