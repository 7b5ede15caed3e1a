"""The C-ABI library loads and exports every entry point declared in
include/*.h; argument errors the reference panics on are reported before any
device work (these run without a GPU)."""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names.update(re.findall(r"GOFFT_API\s+[\w\s\*]+?\b(gofft_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    import fft_b200
    lib = fft_b200.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", fft_b200.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (gofft_\w+)", out))
    decl = declared_symbols()
    assert len(decl) >= 36
    missing = decl - exported
    assert not missing, missing
    for name in decl:
        assert hasattr(lib, name)


def test_python_signatures_cover_header():
    from fft_b200._lib import SIGNATURES
    assert declared_symbols() <= set(SIGNATURES)


def test_version():
    from fft_b200._lib import lib
    assert lib().gofft_version().decode().startswith("gofft-b200")


def test_shape_panics():
    # ndfft_test.go:178-197 and rfft2_test.go:125-146: same panic texts
    from fft_b200 import gofft as G
    with pytest.raises(G.GoPanic, match="shape product does not match"):
        G.FFTN(np.zeros(10, complex), [3, 4])
    with pytest.raises(G.GoPanic, match="shape lengths must be positive"):
        G.FFTN(np.zeros(0, complex), [0, 4])
    with pytest.raises(G.GoPanic, match="shape lengths must be positive"):
        G.FFTN(np.zeros(4, complex), [-1, 4])
    with pytest.raises(G.GoPanic, match="shape lengths must be positive"):
        G.RFFT2(np.zeros(4), [0, 4])
    with pytest.raises(G.GoPanic, match="shape lengths must be positive"):
        G.RFFT2(np.zeros(4), [2, -4])
    with pytest.raises(G.GoPanic, match="shape product does not match"):
        G.RFFT2(np.zeros(5), [2, 4])
    with pytest.raises(G.GoPanic, match="shape lengths must be positive"):
        G.IRFFT2(np.zeros(4, complex), [0, 4])
    with pytest.raises(G.GoPanic, match="shape lengths must be positive"):
        G.IRFFT2(np.zeros(4, complex), [2, -4])


def test_spectrogram_panics():
    # freq_test.go:186-209
    from fft_b200 import gofft as G
    with pytest.raises(G.GoPanic, match="segment length must be positive"):
        G.Spectrogram(np.zeros(0), 0, 0, np.zeros(0), 1)
    with pytest.raises(G.GoPanic, match="window length must equal segment length"):
        G.Spectrogram(np.zeros(0), 4, 0, np.zeros(3), 1)
    with pytest.raises(G.GoPanic, match="overlap must satisfy"):
        G.Spectrogram(np.zeros(0), 4, -1, np.zeros(4), 1)
    with pytest.raises(G.GoPanic, match="overlap must satisfy"):
        G.Spectrogram(np.zeros(0), 4, 4, np.zeros(4), 1)


def test_host_only_edge_cases():
    # fft_test.go:148-168, rfft_test.go:171-183: empty and length-1 inputs
    # never reach the device
    from fft_b200 import gofft as G
    assert G.FFT(np.zeros(0, complex)).size == 0
    assert G.IFFT(np.zeros(0, complex)).size == 0
    one = np.array([7 - 3j])
    assert G.FFT(one)[0] == one[0] and G.IFFT(one)[0] == one[0]
    assert G.RFFT(np.zeros(0)).size == 0
    assert G.IRFFT(np.array([1 + 0j]), 0).size == 0
    assert G.IRFFT(np.array([1 + 0j]), -3).size == 0
    assert G.PSD(np.zeros(0), 1).size == 0
    assert G.Spectrogram(np.array([1.0, 2, 3]), 8, 0, np.ones(8), 1.0) is None
    np.testing.assert_allclose(G.Hann(5), [0, 0.5, 1, 0.5, 0], atol=1e-15)
    assert G.Hann(0).size == 0 and list(G.Hann(1)) == [1]
    sc = G.FFTN(np.array([3 - 2j]), [])
    assert sc.size == 1 and sc[0] == 3 - 2j


def test_wisdom_roundtrip():
    """Wisdom import/export is host logic: entries set, listed and cleared."""
    import json
    from fft_b200 import tune
    from fft_b200._lib import GoFFTError, lib
    tune.forget_wisdom()
    w = {"gofft_wisdom": 1, "schedule": [[0, 512, 1], [2, 1024, 1]], "lpc": [[0, 1024, 0, 1, 8]],
         "pipe": [[1, 256, 0, 1]], "uneven": [[2, 0]]}
    tune.import_wisdom(w)
    got = json.loads(tune.export_wisdom())
    assert sorted(got["schedule"]) == sorted(w["schedule"])
    assert got["lpc"] == w["lpc"] and got["pipe"] == w["pipe"] and got["uneven"] == w["uneven"]
    assert lib().gofft_get_schedule(0, 512) == 1 and lib().gofft_get_schedule(0, 1024) == 0
    for bad in ['{"schedule": [[0, 512, 1]]}', '{"gofft_wisdom":1,"schedule":[[0,512]]}',
                '{"gofft_wisdom":1,"schedule":[[0,512,7]]}', '{"gofft_wisdom":1,"lpc":[[0,1,99,0,4]]}']:
        with pytest.raises(GoFFTError):
            tune.import_wisdom(bad)
    tune.forget_wisdom()
    got = json.loads(tune.export_wisdom())
    assert got["schedule"] == [] and got["lpc"] == [] and got["pipe"] == [] and got["uneven"] == []


def test_host_windows_and_frequencies():
    """The reference-facing windows and bin frequencies (host code, no GPU):
    FFTFreq/RFFTFreq equal numpy's exactly (freq.go:17-56 promises it); the
    windows agree with numpy / scipy and with the oracle's cosine window to
    rounding."""
    import scipy.signal
    from fft_b200 import gofft as G
    from oracle import oracle as O
    for n in [1, 2, 7, 8, 1000, 1001]:
        for d in [1.0, 0.1, 3.7]:
            np.testing.assert_array_equal(G.FFTFreq(n, d), np.fft.fftfreq(n, d))
            np.testing.assert_array_equal(G.RFFTFreq(n, d), np.fft.rfftfreq(n, d))
        assert np.max(np.abs(G.Hamming(n) - np.hamming(n))) < 1e-15
        assert np.max(np.abs(G.Blackman(n) - np.blackman(n))) < 1e-15
        assert np.max(np.abs(G.Bartlett(n) - np.bartlett(n))) < 1e-15
        bh = scipy.signal.windows.blackmanharris(n, sym=True)
        assert np.max(np.abs(G.BlackmanHarris(n) - bh)) < 1e-15
        np.testing.assert_array_equal(G.Hamming(n), O.cosine_window(n, [0.54, 0.46]))
        np.testing.assert_array_equal(G.Blackman(n), O.cosine_window(n, [0.42, 0.5, 0.08]))
    for f in (G.FFTFreq, G.RFFTFreq):
        assert f(0, 1.0).size == 0 and f(-3, 1.0).size == 0
    for f in (G.Hamming, G.Blackman, G.BlackmanHarris, G.Bartlett):
        assert f(0).size == 0 and list(f(1)) == [1.0]
