"""Shared test set-up: the ``gpu`` marker, the package import and golden vectors."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")


@pytest.fixture(scope="session")
def pkg():
    import __graft_entry__ as ge

    return ge.load_package()


@pytest.fixture(scope="session")
def fixtures():
    return dict(np.load(os.path.join(GOLDEN, "fixtures.npz")))


@pytest.fixture(scope="session")
def fft_golden():
    return dict(np.load(os.path.join(GOLDEN, "fft_golden.npz")))


@pytest.fixture(scope="session")
def spectral_golden():
    return dict(np.load(os.path.join(GOLDEN, "spectral_golden.npz")))


def rel_l2(got, want):
    got = np.asarray(got, np.complex128)
    want = np.asarray(want, np.complex128)
    den = np.linalg.norm(want)
    return float(np.linalg.norm(got - want) / (den if den > 0 else 1.0))


def rel_linf(got, want):
    """relError of tests/index.html:89-97: max|got-want| / max|want|."""
    got = np.asarray(got, np.complex128).ravel()
    want = np.asarray(want, np.complex128).ravel()
    num = max(np.max(np.abs(got.real - want.real)), np.max(np.abs(got.imag - want.imag)))
    den = max(np.max(np.abs(want.real)), np.max(np.abs(want.imag)))
    return float(num / den) if den > 0 else float(num)
