"""The oracle (C restatement of go-fft/fft) pinned against the golden
vectors (numpy.fft under the reference's own gate, rtol 1e-9 / atol 1e-7,
benchmarks/verify_correctness.py:16-17) and the reference's known answers."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle as O

RTOL, ATOL = 1e-9, 1e-7


def close(got, want):
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=ATOL)


def test_c2c_golden(golden):
    for k in golden:
        if k.startswith("c2c_in_"):
            n = int(k.split("_")[-1])
            x = golden[k]
            close(O.fft(x), golden["c2c_fft_%d" % n])
            close(O.ifft(x), golden["c2c_ifft_%d" % n])


def test_real_golden(golden):
    for k in golden:
        if k.startswith("r_in_"):
            n = int(k.split("_")[-1])
            close(O.rfft(golden[k]), golden["r_rfft_%d" % n])
            close(O.irfft(golden["r_spec_%d" % n], n), golden["r_irfft_%d" % n])
            close(O.psd(golden[k], 0.25), golden["r_psd_%d" % n])


def test_2d_nd_golden(golden):
    for k in golden:
        if k.startswith("r2_in_"):
            key = k[len("r2_in_"):]
            r, c = map(int, key.split("x"))
            close(O.rfft2(golden[k], r, c).reshape(r, c // 2 + 1), golden["r2_rfft2_" + key])
            back = O.irfft2(O.rfft2(golden[k], r, c), r, c).reshape(r, c)
            close(back, golden["r2_irfft2_" + key])
        if k.startswith("nd_in_"):
            key = k[len("nd_in_"):]
            shape = list(map(int, key.split("x")))
            close(O.fftn(golden[k], shape).reshape(shape), golden["nd_fftn_" + key])
            close(O.ifftn(golden[k], shape).reshape(shape), golden["nd_ifftn_" + key])


# The oracle's own error against numpy.fft / scipy (pocketfft, FP64): far
# inside the 1e-12 budget of the GPU parity tests, so a GPU result within
# 1e-12 of the oracle is within about 1e-12 of an independent FP64 FFT too.
ORACLE_PIN = 1e-13


def test_oracle_pinned_1e13(golden):
    checked = 0
    for k in golden:
        if k.startswith("c2c_in_"):
            n = int(k.split("_")[-1])
            assert rel_l2(O.fft(golden[k]), golden["c2c_fft_%d" % n]) <= ORACLE_PIN, ("fft", n)
            assert rel_l2(O.ifft(golden[k]), golden["c2c_ifft_%d" % n]) <= ORACLE_PIN, ("ifft", n)
            checked += 2
        if k.startswith("r_in_"):
            n = int(k.split("_")[-1])
            assert rel_l2(O.rfft(golden[k]), golden["r_rfft_%d" % n]) <= ORACLE_PIN, ("rfft", n)
            assert rel_l2(O.irfft(golden["r_spec_%d" % n], n), golden["r_irfft_%d" % n]) <= ORACLE_PIN, ("irfft", n)
            checked += 2
        if k.startswith("r2_in_"):
            key = k[len("r2_in_"):]
            r, c = map(int, key.split("x"))
            got = O.rfft2(golden[k], r, c).reshape(r, c // 2 + 1)
            assert rel_l2(got, golden["r2_rfft2_" + key]) <= ORACLE_PIN, ("rfft2", key)
            checked += 1
        if k.startswith("nd_in_"):
            key = k[len("nd_in_"):]
            shape = list(map(int, key.split("x")))
            assert rel_l2(O.fftn(golden[k], shape).reshape(shape), golden["nd_fftn_" + key]) <= ORACLE_PIN
            assert rel_l2(O.ifftn(golden[k], shape).reshape(shape), golden["nd_ifftn_" + key]) <= ORACLE_PIN
            checked += 2
    assert rel_l2(O.spectrogram(golden["spec_in"], 32, 20, golden["spec_win"], 1.0), golden["spec_out"]) <= ORACLE_PIN
    assert checked >= 20


def test_spectrogram_golden(golden):
    got = O.spectrogram(golden["spec_in"], 32, 20, golden["spec_win"], 1.0)
    close(got, golden["spec_out"])


def test_known_answers(kat):
    assert list(O.bit_reverse_perm(8)) == kat["bit_reverse_8"]["value"]
    for p, g in kat["primitive_root"]["value"].items():
        assert O.primitive_root(int(p)) == g
    for n, f in kat["factorize"]["value"].items():
        assert O.factorize(int(n)) == f
    for n, v in kat["factors_small"]["value"].items():
        assert O.factors_small(int(n)) == v
    for n, v in kat["is_prime"]["value"].items():
        assert O.is_prime(int(n)) == v
    assert O.ENGINE_NAMES[O.engine(641)] == "bluestein"
    assert O.ENGINE_NAMES[O.engine(769)] == "rader"
    for n in kat["rader_cyclic"]["value"]:
        info = O.rader_info(n)
        assert info["cyclic"] and info["cl"] == n - 1
    for n in kat["rader_linear"]["value"]:
        info = O.rader_info(n)
        assert not info["cyclic"] and info["cl"] >= 2 * (n - 1) and O.conv_cost(info["cl"])[1]
    for m in kat["conv_cost_not_ok"]["value"]:
        assert not O.conv_cost(m)[1]
    for m in kat["conv_cost_ok"]["value"]:
        assert O.conv_cost(m)[1]
    assert O.rader_info(10007)["cl"] == kat["rader_10007_cl"]["value"]
    np.testing.assert_allclose(O.hann(5), kat["hann_5"]["value"], atol=1e-15)
    assert O.spectrogram(np.sin(np.arange(20.0)), 8, 4, O.hann(8), 1.0).shape[0] == 4


def test_best_conv_len_is_argmin():
    # radix7_test.go:153-184: bestConvLen is the argmin of convCost over its window
    for lo in [1, 2, 16, 10004, 19944, 20012, 100000]:
        g = O.best_conv_len(lo)
        gc, ok = O.conv_cost(g)
        assert ok and g >= lo
        hi = lo + (lo * 4 + 9) // 10
        for m in range(lo, hi + 1):
            c, ok2 = O.conv_cost(m)
            assert not (ok2 and c < gc)


def test_rader_tables_are_permutations():
    for p in [769, 1009, 2017, 10007]:
        info = O.rader_info(p)
        q = p - 1
        assert sorted(info["perm"]) == list(range(1, p))
        assert sorted(info["iperm"]) == list(range(1, p))
        # iperm[q] = perm[(q - qi) mod q] (rader.go:72-74)
        for qi in range(0, q, 97):
            assert info["iperm"][qi] == info["perm"][(q - qi) % q]


def test_chirp_index():
    for n in [17, 641, 1000, 10007]:
        jj = O.chirp_index(n)
        j = np.arange(n, dtype=np.int64)
        assert np.array_equal(jj, (j * j) % (2 * n))


def test_engines_cross_check():
    # rader_test.go:80-96: Rader and Bluestein agree on the large primes
    g = np.random.default_rng(7)
    for n in [769, 1009, 2017, 10007]:
        x = g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)
        a = O.rader(x)
        b = O.bluestein(x)
        # the reference's tolerance: max |diff| <= 1e-13 n^2 (rader_test.go:22)
        assert np.max(np.abs(a - b)) <= 1e-13 * n * n
        assert rel_l2(a, np.fft.fft(x)) < 1e-13


def test_naive_dft_small():
    # fft_test.go:12-24: O(N^2) DFT oracle for small n
    for n in range(1, 40):
        x = np.sin(np.arange(n) * 0.7) + (np.arange(n) % 3) + 1j * np.cos(np.arange(n) * 0.3)
        k = np.arange(n)
        naive = (x[None, :] * np.exp(-2j * np.pi * np.outer(k, k) / n)).sum(axis=1)
        assert np.max(np.abs(O.fft(x) - naive)) < 1e-9


@pytest.mark.parametrize("workers", [1, 3, 8])
def test_parallel_matches_serial(workers):
    # parallel_test.go:64-106: worker count never changes results
    g = np.random.default_rng(3)
    x = g.standard_normal((64, 300))
    O.set_workers(1)
    a = O.rfft2(x, 64, 300)
    O.set_workers(workers)
    b = O.rfft2(x, 64, 300)
    O.set_workers(0)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("shape", [(16,), (15,), (1,), (2,), (8, 6), (7, 5), (1, 9), (6, 1)])
def test_adjoint_identities(shape):
    """The identities the adjoint kernels implement, checked as dot-product
    tests on the oracle's transforms (real inner product Re sum conj(a) b):
    RFFT^T(G) = N IRFFT(G / w) and IRFFT^T(g) = (w / N) RFFT(g), w the
    edge-bin weights of the last axis; FFT^H = N IFFT."""
    from conftest import edge_weights, rdot, rng
    g = rng(11)
    N = int(np.prod(shape))
    cols = shape[-1]
    K = cols // 2 + 1
    bshape = shape[:-1] + (K,)
    w = edge_weights(cols)
    if len(shape) == 1:
        fwd = lambda v: O.rfft(v)
        inv = lambda S: O.irfft(S, cols)
    else:
        fwd = lambda v: O.rfft2(v, *shape).reshape(bshape)
        inv = lambda S: O.irfft2(S, *shape).reshape(shape)
    for _ in range(3):
        x = g.standard_normal(shape)
        G = g.standard_normal(bshape) + 1j * g.standard_normal(bshape)
        lhs = rdot(fwd(x), G)
        rhs = rdot(x, N * inv(G / w))
        assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + np.linalg.norm(x) * np.linalg.norm(G))
        y = g.standard_normal(shape)
        lhs = rdot(inv(G), y)
        rhs = rdot(G, w / N * fwd(y))
        assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + np.linalg.norm(y) * np.linalg.norm(G))
    z = g.standard_normal(N) + 1j * g.standard_normal(N)
    Z = g.standard_normal(N) + 1j * g.standard_normal(N)
    cs = list(shape)
    assert abs(rdot(O.fftn(z, cs), Z) - rdot(z, N * O.ifftn(Z, cs))) <= 1e-12 * N * np.linalg.norm(z) * np.linalg.norm(Z)


def test_filter_gradient_identity():
    """dx and dH of L = sum(y^2), y = IRFFT2(H * RFFT2(x)), as assembled from
    the oracle's transforms, against central differences on a small case
    (L is quadratic, so the central difference is exact up to rounding)."""
    from conftest import filter_case, filter_oracle, rng
    x, H = filter_case(batch=2, rows=6, cols=8)
    x = x.astype(np.float64)
    H = H.astype(np.complex128)
    y, dx, dH = filter_oracle(x, H)
    loss = lambda xx, HH: float(np.sum(filter_oracle(xx, HH)[0] ** 2))
    e = 1e-6
    g = rng(3)
    for _ in range(8):
        b, i, j = g.integers(0, 2), g.integers(0, 6), g.integers(0, 8)
        xp, xm = x.copy(), x.copy()
        xp[b, i, j] += e
        xm[b, i, j] -= e
        fd = (loss(xp, H) - loss(xm, H)) / (2 * e)
        assert abs(fd - dx[b, i, j]) <= 1e-6 * (1 + abs(dx[b, i, j]))
        r, k = g.integers(0, 6), g.integers(0, 5)
        for unit in (1.0, 1j):
            Hp, Hm = H.copy(), H.copy()
            Hp[r, k] += e * unit
            Hm[r, k] -= e * unit
            fd = (loss(x, Hp) - loss(x, Hm)) / (2 * e)
            want = dH[r, k].real if unit == 1.0 else dH[r, k].imag
            assert abs(fd - want) <= 1e-6 * (1 + abs(want))
