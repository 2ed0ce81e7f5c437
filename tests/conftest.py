"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device and the built libexo_b200.so; all
others run on the CPU.  The CPU oracle (oracle/) is the checker of the GPU
path and is built on demand.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def native():
    from exocubed_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        _native.build()
    _native.lib()
    return _native
