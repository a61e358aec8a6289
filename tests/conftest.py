"""Shared test setup: the `gpu` marker, repository paths and fixtures.

Tests marked `gpu` need a CUDA device and call the library through its C ABI; the others run on the CPU (oracle
against the golden fixtures, host logic, ABI exports).
"""
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "case_*.npz")))


@pytest.fixture(scope="session")
def oracle():
    from pyoracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def known():
    return dict(np.load(os.path.join(GOLDEN, "known_answers.npz")))


@pytest.fixture(scope="session")
def ctx():
    import ryoanji_b200 as ryo
    return ryo.Context(0)
