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


def rdot(a, b):
    """Real inner product Re sum conj(a) b (the one the adjoints use)."""
    a = np.asarray(a).astype(np.complex128).ravel()
    b = np.asarray(b).astype(np.complex128).ravel()
    return float(np.real(np.vdot(a, b)))


def edge_weights(cols):
    """Real-spectrum edge-bin weights along an axis of `cols` reals:
    1 at bin 0 and bin cols/2 (even cols), 2 elsewhere."""
    w = np.full(cols // 2 + 1, 2.0)
    w[0] = 1.0
    if cols % 2 == 0:
        w[-1] = 1.0
    return w


def filter_case(batch=32, rows=512, cols=512, seed_x=4, seed_h=5):
    """The differentiation workload: x float32 (batch, rows, cols) uniform
    [0, 1) from seed_x; H complex64 (rows, cols/2+1), a Gaussian low-pass
    exp(-(kr^2 + kc^2) / (2 * 40^2)) (kr the signed row frequency, kc the
    column bin) times exp(i phi), phi uniform [0, 2 pi) from seed_h."""
    x = np.random.default_rng(seed_x).random((batch, rows, cols), dtype=np.float32)
    kr = np.fft.fftfreq(rows, 1.0 / rows)[:, None]
    kc = np.arange(cols // 2 + 1)[None, :]
    mag = np.exp(-(kr ** 2 + kc ** 2) / (2.0 * 40.0 ** 2))
    phi = np.random.default_rng(seed_h).uniform(0.0, 2.0 * np.pi, (rows, cols // 2 + 1))
    H = (mag * np.exp(1j * phi)).astype(np.complex64)
    return x, H


def filter_oracle(x, H, g=None):
    """Forward y_b = IRFFT2(H * RFFT2(x_b)) and the gradients of
    L = sum(y^2) (or of <y, g> when g is given) assembled from the oracle's
    transforms:  dx = IRFFT2(conj(H) * RFFT2(gy)),
    dH = sum_b conj(X_b) * (w / (R C)) * RFFT2(gy_b),  gy = 2y or g."""
    from oracle import oracle as O
    B, R, C = x.shape
    K = C // 2 + 1
    Hc = np.asarray(H, np.complex128).reshape(R, K)
    w = edge_weights(C)[None, :] / float(R * C)
    y = np.zeros((B, R, C))
    dx = np.zeros((B, R, C))
    dH = np.zeros((R, K), np.complex128)
    for b in range(B):
        X = O.rfft2(x[b].astype(np.float64), R, C).reshape(R, K)
        y[b] = O.irfft2(Hc * X, R, C).reshape(R, C)
        gy = 2.0 * y[b] if g is None else np.asarray(g[b], np.float64)
        G = O.rfft2(gy, R, C).reshape(R, K)
        dx[b] = O.irfft2(np.conj(Hc) * G, R, C).reshape(R, C)
        dH += np.conj(X) * w * G
    return y, dx, dH
