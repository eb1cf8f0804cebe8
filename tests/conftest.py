"""Shared test set-up.

Markers: ``gpu`` tests need a CUDA device and run the drop-in through its C
ABI; everything else runs on the CPU (oracle, host set-up, ABI exports,
multi-process host logic).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session", autouse=True)
def _native_libs():
    """Build the host library and the oracle if they are missing (CPU-only
    work); the CUDA library is built by __graft_entry__.build()."""
    from sddc_b200 import build

    build.build_host()
    build.build_oracle()
    yield
