"""Shared pytest setup: the `gpu` marker, import paths and module fixtures.

CPU tests (``-m "not gpu"``) cover the oracle against the known-answer
fixtures, the host logic and the C-ABI surface; ``-m gpu`` tests run the CUDA
engines on a B200 and compare them with the oracle through the C-ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "tensor-episdet_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def episdet():
    import episdet as m

    m.lib()
    return m


@pytest.fixture(scope="session")
def oracle():
    import pyoracle as m

    m.build()
    m.lib()
    return m
