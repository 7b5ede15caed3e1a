"""Spectral helpers on the GPU: device-generated windows against the
reference-facing host windows, the spectrogram with a device window against
the oracle, and go-fft's parity-harness document produced by this engine,
checked the way go-fft's own correctness gate checks it (numpy.fft,
rtol 1e-9, atol 1e-7)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KINDS = ["hann", "hamming", "blackman", "blackmanharris", "bartlett"]


def host_window(kind, n):
    from fft_b200 import gofft as G
    return {"hann": G.Hann, "hamming": G.Hamming, "blackman": G.Blackman, "blackmanharris": G.BlackmanHarris,
            "bartlett": G.Bartlett}[kind](n)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [1, 2, 5, 64, 2047, 2048])
def test_device_windows(kind, n):
    from fft_b200.device import window
    want = host_window(kind, n)
    got64 = window(kind, n, "f64").cpu().numpy()
    assert np.max(np.abs(got64 - want)) <= 2e-15
    got32 = window(kind, n, "f32").cpu().numpy()
    assert np.max(np.abs(got32.astype(np.float64) - want)) <= 1e-7


@pytest.mark.parametrize("kind", ["hamming", "blackmanharris"])
@pytest.mark.parametrize("prec", ["f64", "f32mixed"])
def test_spectrogram_device_window(kind, prec):
    from fft_b200.device import spectrogram_window
    x = rng(8).standard_normal(1 << 15)
    rdt = torch.float64 if prec == "f64" else torch.float32
    xt = torch.from_numpy(x).to(rdt).cuda()
    got = spectrogram_window(xt, 1024, 768, kind, 0.5, prec).cpu().numpy()
    want = O.spectrogram(xt.cpu().numpy().astype(np.float64), 1024, 768, host_window(kind, 1024), 0.5)
    assert got.shape == want.shape
    assert rel_l2(got, want) <= (1e-12 if prec == "f64" else 1e-6)


def test_parity_harness_document():
    from fft_b200 import verify as V
    doc = V.dump()
    assert sorted(doc) == ["complex", "fft2", "ireal", "real"]
    ok = lambda got, ref: np.allclose(got, ref, rtol=1e-9, atol=1e-7)
    to_np = lambda pairs: np.array([p["Re"] + 1j * p["Im"] for p in pairs])
    for k, pairs in doc["complex"].items():
        assert ok(to_np(pairs), np.fft.fft(V.cmplx(int(k)))), k
    for k, pairs in doc["real"].items():
        assert ok(to_np(pairs), np.fft.rfft(V.realv(int(k)))), k
    for k, vals in doc["ireal"].items():
        assert ok(np.asarray(vals), np.fft.irfft(V.halfspec(int(k)), int(k))), k
    for k, pairs in doc["fft2"].items():
        a, b = (int(v) for v in k.split("x"))
        assert ok(to_np(pairs).reshape(a, b), np.fft.fft2(V.cmplx(a * b).reshape(a, b))), k
    assert len(doc["complex"]) == 9 and len(doc["real"]) == 6 and len(doc["fft2"]) == 3
