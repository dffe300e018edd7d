"""Shared pytest setup: the `gpu` marker and import paths.

GPU tests (marked `gpu`) call the CUDA library through its C-ABI and compare
against the CPU oracle (oracle/, test infrastructure only).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libcosa_gpu.so")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle
