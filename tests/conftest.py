"""Test configuration: the `gpu` marker, import paths and shared fixtures.

`-m "not gpu"` runs on any host: the oracle against the golden fixtures, the
host-side DAG logic and the C-ABI exports.  `-m gpu` runs the parity tests on a
B200 through the C ABI of libchameleon_b200.so.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def cb():
    import chameleon_b200 as cb
    cb.init()
    return cb


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    return oracle
