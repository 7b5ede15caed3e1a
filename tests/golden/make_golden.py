"""Generates the committed golden fixtures in this directory.

    python tests/golden/make_golden.py

* ``vectors.npz`` -- seeded inputs (numpy PCG64) and numpy.fft / scipy
  outputs for small transforms of every engine class.  numpy.fft (pocketfft)
  is the independent implementation the reference's own parity gate checks
  go-fft against (benchmarks/verify_correctness.py:16-17, rtol 1e-9,
  atol 1e-7); the oracle is pinned to these vectors with that gate.
* ``kat.json`` -- known-answer values from the reference's unit tests, with
  the test file:line each comes from.

The go-fft reference ships no output vectors of its own (its benchmarks/*.json
hold timings only), and no Go toolchain exists to run it here.
"""
import json
import os

import numpy as np
import scipy.signal

HERE = os.path.dirname(os.path.abspath(__file__))

C2C_LENGTHS = list(range(1, 65)) + [60, 96, 100, 121, 128, 169, 289, 360, 641, 769, 1000, 1008, 1009, 1024,
                                    1296, 2017, 2018, 4096, 10007]
REAL_LENGTHS = list(range(1, 41)) + [64, 100, 128, 1000, 1024, 2048, 2018]
R2_SHAPES = [(4, 6), (3, 5), (2, 8), (5, 4), (1, 1), (7, 3), (1, 6), (6, 1), (16, 16), (64, 48), (33, 17)]
ND_SHAPES = [(2, 2), (3, 4), (4, 3), (1, 5), (5, 1), (2, 3, 4), (3, 1, 2), (2, 2, 2, 2), (6, 5), (8, 6, 10)]


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    for n in C2C_LENGTHS:
        x = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        out["c2c_in_%d" % n] = x
        out["c2c_fft_%d" % n] = np.fft.fft(x)
        out["c2c_ifft_%d" % n] = np.fft.ifft(x)
    for n in REAL_LENGTHS:
        x = rng.standard_normal(n)
        out["r_in_%d" % n] = x
        out["r_rfft_%d" % n] = np.fft.rfft(x)
        h = rng.standard_normal(n // 2 + 1) + 1j * rng.standard_normal(n // 2 + 1)
        out["r_spec_%d" % n] = h
        out["r_irfft_%d" % n] = np.fft.irfft(h, n)
        out["r_psd_%d" % n] = scipy.signal.periodogram(x, fs=1.0 / 0.25, window="boxcar", scaling="density", detrend=False)[1]
    for s in R2_SHAPES:
        x = rng.standard_normal(s)
        key = "%dx%d" % s
        out["r2_in_" + key] = x
        out["r2_rfft2_" + key] = np.fft.rfft2(x)
        out["r2_irfft2_" + key] = np.fft.irfft2(np.fft.rfft2(x), s)
    for s in ND_SHAPES:
        x = rng.standard_normal(s) + 1j * rng.standard_normal(s)
        key = "x".join(map(str, s))
        out["nd_in_" + key] = x
        out["nd_fftn_" + key] = np.fft.fftn(x)
        out["nd_ifftn_" + key] = np.fft.ifftn(x)
    # spectrogram: each frame is the periodogram of its Hann-windowed segment
    x = rng.standard_normal(300)
    seg, ov = 32, 20
    w = np.hanning(seg)
    frames = [scipy.signal.periodogram(x[t:t + seg] * w, fs=1.0, window="boxcar", scaling="density", detrend=False)[1]
              for t in range(0, len(x) - seg + 1, seg - ov)]
    out["spec_in"] = x
    out["spec_win"] = w
    out["spec_out"] = np.array(frames)
    np.savez_compressed(os.path.join(HERE, "vectors.npz"), **out)

    kat = {
        "bit_reverse_8": {"value": [0, 4, 2, 6, 1, 5, 3, 7], "ref": "internal/kernels/kernels_test.go:21-31"},
        "primitive_root": {"value": {"2": 1, "3": 2, "5": 2, "7": 3, "11": 2, "13": 2, "17": 3, "23": 5},
                           "ref": "rader_test.go:130-149"},
        "factorize": {"value": {"16": [4, 4], "8": [4, 2], "12": [4, 3], "1296": [4, 4, 3, 3, 3, 3],
                                "1000": [4, 2, 5, 5, 5], "13": [13]}, "ref": "plan_test.go:102-126"},
        "factors_small": {"value": {"169": True, "17": False, "34": False}, "ref": "plan_test.go:127-136"},
        "is_prime": {"value": {"0": False, "1": False, "2": True, "3": True, "4": False, "9": False, "17": True,
                               "25": False, "10007": True, "10006": False, "9973": True},
                     "ref": "rader_test.go:152-162"},
        "routing": {"value": {"641": "bluestein", "769": "rader"}, "ref": "rader_test.go:165-180"},
        "rader_cyclic": {"value": [769, 2017], "ref": "radix7_test.go:109-117"},
        "rader_linear": {"value": [5003, 9973, 10007], "ref": "radix7_test.go:118-130"},
        "conv_cost_not_ok": {"value": [11, 22, 121, 554, 5003, 10006], "ref": "radix7_test.go:134-140"},
        "conv_cost_ok": {"value": [1, 2, 4, 8, 7, 10080, 20580, 21952], "ref": "radix7_test.go:141-151"},
        "hann_5": {"value": [0, 0.5, 1, 0.5, 0], "ref": "window_test.go:41-45"},
        "spectrogram_frames_20_8_4": {"value": 4, "ref": "freq_test.go:150-163"},
        "rader_10007_cl": {"value": 20580, "ref": "plan.go:192-259 (convCost/bestConvLen; plan.go:239-240)"},
    }
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
