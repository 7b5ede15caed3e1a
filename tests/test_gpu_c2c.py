"""Complex transforms on the B200 against the oracle (the C restatement of
go-fft/fft): FP64 within relative L2 1e-12, the FP32 forms within 1e-6.
Lengths cover every engine: single-CTA Stockham (powers of two and 13-smooth
composites), the two-pass four-step split, Rader (cyclic and padded-linear,
fused and multi-pass) and Bluestein."""
import numpy as np
import pytest
import torch

from conftest import rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
F32_TOL = 1e-6

POW2 = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 65536]
SMOOTH = [3, 5, 6, 7, 9, 11, 12, 13, 15, 60, 100, 121, 169, 360, 1000, 1008, 1296, 2310, 20580]
PRIMES = [17, 19, 23, 31, 641, 769, 1009, 2017, 9973, 10007]
BLUE = [34, 46, 289, 2018, 3 * 1009]


def sig(n, seed):
    g = rng(seed)
    return g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)


@pytest.mark.parametrize("n", POW2 + SMOOTH + PRIMES + BLUE)
def test_plan_fft_ifft_f64(n):
    from fft_b200 import gofft as G
    x = sig(n, n)
    p = G.NewPlan(n)
    assert p.Len() == n
    X = p.FFT(np.zeros(n, complex), x)
    assert rel_l2(X, O.fft(x)) <= F64_TOL
    back = p.IFFT(np.zeros(n, complex), X)
    assert rel_l2(back, O.ifft(X)) <= F64_TOL
    assert np.max(np.abs(back - x)) < 1e-9


def test_trivial_and_alias():
    # plan_test.go:70-98, fft_test.go:148-184
    from fft_b200 import gofft as G
    p0 = G.NewPlan(0)
    assert p0.FFT(np.zeros(0, complex), np.zeros(0, complex)).size == 0
    one = np.array([7 - 3j])
    p1 = G.NewPlan(1)
    assert p1.FFT(np.zeros(1, complex), one)[0] == one[0]
    assert p1.IFFT(np.zeros(1, complex), one)[0] == one[0]
    for n in [8, 12, 1296, 23, 10007]:
        x = sig(n, 5)
        want = O.fft(x)
        G.NewPlan(n).FFT(x, x)  # in place
        assert rel_l2(x, want) <= F64_TOL
    x = sig(10, 9)
    orig = x.copy()
    G.FFT(x)
    G.IFFT(x)
    assert np.array_equal(x, orig)


def test_known_answers():
    # fft_test.go:63-134: impulse, constant, sinusoid, linearity
    from fft_b200 import gofft as G
    for n in [4, 6, 8, 13, 9, 15, 25, 23, 49, 769]:
        x = np.zeros(n, complex)
        x[0] = 1
        assert np.max(np.abs(G.FFT(x) - 1)) < 1e-9
    for n in [4, 7, 8, 1009]:
        X = G.FFT(np.ones(n, complex))
        want = np.zeros(n, complex)
        want[0] = n
        assert np.max(np.abs(X - want)) < 1e-9
    n, f = 16, 3
    X = G.FFT(np.exp(2j * np.pi * f * np.arange(n) / n))
    mag = np.abs(X)
    assert abs(mag[f] - n) < 1e-9 and np.all(np.delete(mag, f) < 1e-9)
    n = 10
    a, b = 2 - 1j, 0.5 + 3j
    x = np.arange(n) - 0.2j * np.arange(n)
    y = np.cos(np.arange(n)) + 1j * (np.arange(n) % 4)
    assert np.max(np.abs(G.FFT(a * x + b * y) - (a * G.FFT(x) + b * G.FFT(y)))) < 1e-9


def test_cached_plan_identity():
    # radix7_test.go:13-41: the cache returns one plan per length
    from fft_b200 import gofft as G
    a = G.cachedPlan(9973)
    b = G.cachedPlan(9973)
    assert a._h.value == b._h.value


def test_batched_config1_roundtrip():
    # 256 complex128 signals of length 1024, uniform[-1,1) from seed 0
    from fft_b200.device import DevicePlan
    g = np.random.default_rng(0)
    x = g.uniform(-1, 1, (256, 1024)) + 1j * g.uniform(-1, 1, (256, 1024))
    p = DevicePlan("c2c", "f64", [1024], batch=256)
    X = p.c2c(torch.from_numpy(x).cuda())
    want = O.batch_fft(x)
    assert rel_l2(X.cpu().numpy(), want) <= F64_TOL
    back = p.c2c(X, inverse=True)
    assert rel_l2(back.cpu().numpy(), O.batch_fft(want, inverse=True)) <= F64_TOL
    assert np.max(np.abs(back.cpu().numpy() - x)) < 1e-12


@pytest.mark.parametrize("n", [1000, 65536, 10007, 2018, 1009])
def test_batched_strided(n):
    # element i of transform b at b*idist + i*istride
    from fft_b200.device import DevicePlan
    B, st = 3, 2
    x = sig(B * n * st + 5, 11).astype(np.complex128)
    p = DevicePlan("c2c", "f64", [n], batch=B, istride=st, idist=n * st + 1, ostride=1, odist=n)
    out = torch.zeros(B * n, dtype=torch.complex128, device="cuda")
    p.c2c(torch.from_numpy(x).cuda(), out=out)
    got = out.cpu().numpy().reshape(B, n)
    for b in range(B):
        assert rel_l2(got[b], O.fft(x[b * (n * st + 1):][: n * st:st])) <= F64_TOL


@pytest.mark.parametrize("prec", ["f32", "f32mixed"])
@pytest.mark.parametrize("n", [60, 128, 360, 1000, 1009, 4096, 10007, 65536, 2018, 20580])
def test_fp32_forms(prec, n):
    from fft_b200.device import DevicePlan
    B = 4
    g = rng(n + 1)
    x = (g.uniform(-1, 1, (B, n)) + 1j * g.uniform(-1, 1, (B, n))).astype(np.complex64)
    p = DevicePlan("c2c", prec, [n], batch=B)
    X = p.c2c(torch.from_numpy(x).cuda()).cpu().numpy()
    want = O.batch_fft(x.astype(np.complex128))
    err = rel_l2(X, want)
    assert err <= F32_TOL, err
    back = p.c2c(torch.from_numpy(X).cuda(), inverse=True).cpu().numpy()
    assert rel_l2(back, x.astype(np.complex128)) <= 2 * F32_TOL


def test_mixed_beats_plain_fp32_on_long_lengths():
    # hi+lo twiddles remove the twiddle rounding error of the plain FP32 form
    from fft_b200.device import DevicePlan
    n, B = 65536, 8
    g = rng(2)
    x = (g.uniform(-1, 1, (B, n)) + 1j * g.uniform(-1, 1, (B, n))).astype(np.complex64)
    want = O.batch_fft(x.astype(np.complex128))
    e = {}
    for prec in ["f32", "f32mixed"]:
        X = DevicePlan("c2c", prec, [n], batch=B).c2c(torch.from_numpy(x).cuda()).cpu().numpy()
        e[prec] = rel_l2(X, want)
    assert e["f32mixed"] <= e["f32"]


def test_integer_tables_bit_exact():
    from fft_b200.device import DevicePlan
    for p in [769, 1009, 2017, 10007]:
        plan = DevicePlan("c2c", "f64", [p])
        info = O.rader_info(p)
        assert plan.table(3) == [info["g"], info["cl"]]
        assert plan.table(0) == list(info["perm"])
        assert plan.table(1) == list(info["iperm"])
    for n in [17, 641, 2018, 289]:
        plan = DevicePlan("c2c", "f64", [n])
        assert plan.table(4) == [O.bluestein_m(n)]
        assert plan.table(2) == list(O.chirp_index(n))


def test_routing_matches_reference():
    from fft_b200.device import DevicePlan
    assert DevicePlan("c2c", "f64", [641]).describe()["axes"][0]["engine"] == "bluestein"
    assert DevicePlan("c2c", "f64", [769]).describe()["axes"][0]["engine"] == "rader"
    d = DevicePlan("c2c", "f64", [10007]).describe()["axes"][0]
    assert d["engine"] == "rader" and d["cl"] == 20580 and d["cyclic"] == 0
    d = DevicePlan("c2c", "f64", [1009]).describe()["axes"][0]
    assert d["cl"] == 1008 and d["cyclic"] == 1
    assert DevicePlan("c2c", "f64", [1024]).describe()["axes"][0]["engine"] == "single"
    assert DevicePlan("c2c", "f64", [65536]).describe()["axes"][0]["engine"] == "fourstep"


SAME = {"f64": 2e-15, "f32mixed": 2e-7}


@pytest.mark.parametrize("prec", ["f64", "f32mixed"])
def test_fourstep_l2_blocks_on_lanes(prec):
    """A batched four-step plan split into L2 blocks of signals on two lanes
    (1 MiB budget: one 65536-point FP64 signal, two FP32 ones per block), from
    a strided layout with gaps between signals, in place and out of place:
    equal to the unblocked plan (the lines per CTA follow each launch's line
    count, so a block may run other kernel instances: the same arithmetic up
    to the compiler's fused multiply-adds) and to the oracle."""
    from fft_b200 import tune
    from fft_b200.device import DevicePlan
    n, B, gap = 65536, 7, 3
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    g = rng(41)
    x = torch.from_numpy(g.standard_normal(B * (n + gap)) + 1j * g.standard_normal(B * (n + gap))).to(cdt).cuda()
    tune.set_l2_block_bytes(1 << 20)
    try:
        p = DevicePlan("c2c", prec, [n], batch=B, idist=n + gap, odist=n + gap)
    finally:
        tune.set_l2_block_bytes(0)
    tune.set_lanes(1)
    try:
        q = DevicePlan("c2c", prec, [n], batch=B, idist=n + gap, odist=n + gap)
    finally:
        tune.set_lanes(0)
    assert p.describe()["line_blocks"] == (1 if prec == "f64" else 2) and q.describe()["line_blocks"] == 0
    for inverse in (False, True):
        got = torch.zeros_like(x)
        want = torch.zeros_like(x)
        p.c2c(x, out=got, inverse=inverse)
        q.c2c(x, out=want, inverse=inverse)
        torch.cuda.synchronize()
        gv, wv = got.cpu().numpy(), want.cpu().numpy()
        assert rel_l2(gv, wv) <= SAME[prec]
        xv = x.cpu().numpy().astype(np.complex128)
        for b in (0, B - 1):
            o = b * (n + gap)
            ref = (O.ifft if inverse else O.fft)(xv[o:o + n])
            assert rel_l2(gv[o:o + n], ref) <= (F64_TOL if prec == "f64" else 1e-6)
    z = x.clone()
    p.c2c(z, out=z)
    w = x.clone()
    q.c2c(w, out=w)
    assert rel_l2(z.cpu().numpy(), w.cpu().numpy()) <= SAME[prec]
