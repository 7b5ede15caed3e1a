"""go-fft's parity-harness output, produced by this engine.

    python -m fft_b200.verify > gpu.json

writes the JSON document go-fft's benchmarks/verify/main.go writes (keys
"complex", "real", "ireal", "fft2"; complex values as {"Re", "Im"} objects),
on the same deterministic inputs and sizes, with every transform computed by
libgofft_b200.so through the Go-API mirror.  go-fft's own correctness gate
(benchmarks/verify_correctness.py, numpy.fft within rtol 1e-9 / atol 1e-7)
reads it unchanged.
"""
import json
import sys

import numpy as np

from . import gofft as G

# verify/main.go's sizes
COMPLEX_SIZES = [256, 1024, 4096, 1000, 1080, 1920, 1009, 1296, 10007]
REAL_SIZES = [256, 1024, 4096, 1000, 1080, 1920]
FFT2_SHAPES = [(64, 64), (128, 128), (256, 256)]


def cmplx(n):
    """The harness's complex input: ((i*7+1) mod 13)/10 + i ((i*3+2) mod 11)/10."""
    i = np.arange(n)
    return ((i * 7 + 1) % 13) * 0.1 + 1j * (((i * 3 + 2) % 11) * 0.1)


def realv(n):
    """The harness's real input: ((i*7+1) mod 13)/10."""
    i = np.arange(n)
    return ((i * 7 + 1) % 13) * 0.1


def halfspec(n):
    """The harness's n/2+1-bin half spectrum for the inverse real transform."""
    return cmplx(n // 2 + 1)


def _pairs(z):
    return [{"Re": float(v.real), "Im": float(v.imag)} for v in np.asarray(z, np.complex128)]


def dump():
    """The harness document as a dict."""
    out = {"complex": {}, "real": {}, "ireal": {}, "fft2": {}}
    for n in COMPLEX_SIZES:
        out["complex"][str(n)] = _pairs(G.FFT(cmplx(n)))
    for n in REAL_SIZES:
        out["real"][str(n)] = _pairs(G.RFFT(realv(n)))
        out["ireal"][str(n)] = [float(v) for v in G.IRFFT(halfspec(n), n)]
    for a, b in FFT2_SHAPES:
        out["fft2"]["%dx%d" % (a, b)] = _pairs(G.FFT2(cmplx(a * b), (a, b)))
    return out


def main():
    json.dump(dump(), sys.stdout)
    sys.stdout.write("\n")


if __name__ == "__main__":
    main()
