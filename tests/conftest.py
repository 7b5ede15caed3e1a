"""Shared test setup: the repo root on sys.path, the `gpu` marker, fixtures.

Tests marked `gpu` need a CUDA device and the built libgofft_b200.so; the
rest run on CPU (oracle vs golden vectors, host logic, library symbols)."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built engine")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "vectors.npz")))


@pytest.fixture(scope="session")
def kat():
    with open(os.path.join(GOLDEN, "kat.json")) as f:
        return json.load(f)


def rel_l2(got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    den = np.linalg.norm(want.astype(np.complex128).ravel())
    num = np.linalg.norm((got.astype(np.complex128) - want.astype(np.complex128)).ravel())
    return num / den if den > 0 else num


def rng(seed):
    return np.random.default_rng(seed)
