"""Test configuration: the `gpu` marker, import paths and shared fixtures.

`-m "not gpu"` runs here without a GPU: oracle vs golden vectors and the
compiled reference, host logic, and the C ABI's exports.  `-m gpu` tests run
the CUDA path through the C ABI and compare it with the oracle.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "squares-in-squares_b200"
for p in (ROOT, PKG, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (runs the CUDA path)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    return O


@pytest.fixture(scope="session")
def ctx():
    from sqs import Context
    c = Context(0)
    yield c
    c.close()
