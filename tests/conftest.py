"""Test configuration: the `gpu` marker, import paths and shared fixtures.

`-m "not gpu"` covers the oracle (against the reference's own known answers), the
host-side mesher and package logic, and that the C-ABI library loads and exports every
entry point of include/tmsolve.h. `-m gpu` holds the parity tests proper: the CUDA path
through the C-ABI against the oracle on the same inputs.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "packaging-tm-modeling-tool_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA path through the C-ABI)")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle
