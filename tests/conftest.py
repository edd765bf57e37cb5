"""Shared pytest set-up: the ``gpu`` marker and import paths.

``-m "not gpu"`` tests run on the CPU (oracle vs golden vectors, host logic,
C-ABI symbol checks); ``-m gpu`` tests call the CUDA path through the C-ABI
and compare it with the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "jax-hfbfft_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
