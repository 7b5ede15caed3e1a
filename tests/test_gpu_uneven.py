"""Uneven batches (many lengths in one persistent launch) and CUDA-graph
replay, against the oracle's per-signal transforms."""
import numpy as np
import pytest
import torch

from conftest import rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C3_LENGTHS = [60, 128, 360, 1000, 1009, 4096, 10007, 65536]
TOL = {"f64": 1e-12, "f32": 1e-6, "f32mixed": 1e-6}


def make_batch(lengths, seed, dtype):
    g = rng(seed)
    parts = [(g.uniform(-1, 1, n) + 1j * g.uniform(-1, 1, n)) for n in lengths]
    flat = np.concatenate(parts).astype(dtype)
    return parts, flat


def check_all(lengths, got, parts, prec, inverse=False, out_offsets=None):
    off = 0
    for i, n in enumerate(lengths):
        o = out_offsets[i] if out_offsets is not None else off
        want = (O.ifft if inverse else O.fft)(parts[i].astype(np.complex128))
        err = rel_l2(got[o:o + n], want)
        assert err <= TOL[prec], (prec, n, err)
        off += n


@pytest.mark.parametrize("prec", ["f64", "f32mixed", "f32"])
@pytest.mark.parametrize("persistent", [1, 0])
def test_uneven_c3_lengths(prec, persistent):
    from fft_b200.device import UnevenBatch
    g = rng(2)
    lengths = [int(C3_LENGTHS[i]) for i in g.integers(0, len(C3_LENGTHS), 40)] + C3_LENGTHS
    dt = np.complex128 if prec == "f64" else np.complex64
    parts, flat = make_batch(lengths, 3, dt)
    u = UnevenBatch(prec, lengths)
    u.set(0, persistent)
    x = torch.from_numpy(flat).cuda()
    y = u(x)
    assert u.status() == 0
    check_all(lengths, y.cpu().numpy(), parts, prec)
    z = u(x, inverse=True)
    assert u.status() == 0
    check_all(lengths, z.cpu().numpy(), parts, prec, inverse=True)
    d = u.describe()
    assert d["items"] > 0 and len(d["classes"]) == len(set(lengths))
    assert d["persistent"] == persistent


@pytest.mark.parametrize("persistent", [1, 0])
def test_uneven_longest_inplace_rader_f64(persistent):
    """13721 in FP64: its cyclic convolution of 13720 complex128 (219 KB) is
    the longest that runs in one CTA's shared memory; the persistent launch
    is sized for the unpadded convolution and still fits an SM."""
    from fft_b200.device import DevicePlan, UnevenBatch
    assert DevicePlan("c2c", "f64", [13721]).describe()["axes"][0]["inplace"] == 1
    lengths = [13721, 64, 13721, 1000, 13721]
    parts, flat = make_batch(lengths, 9, np.complex128)
    u = UnevenBatch("f64", lengths)
    u.set(0, persistent)
    y = u(torch.from_numpy(flat).cuda())
    assert u.status() == 0
    check_all(lengths, y.cpu().numpy(), parts, "f64")


def test_uneven_inplace_and_offsets():
    from fft_b200.device import UnevenBatch
    lengths = [1009, 60, 65536, 17, 641, 10007, 128]
    parts, flat = make_batch(lengths, 5, np.complex128)
    # in place
    u = UnevenBatch("f64", lengths)
    x = torch.from_numpy(flat.copy()).cuda()
    u(x, out=x)
    assert u.status() == 0
    check_all(lengths, x.cpu().numpy(), parts, "f64")
    # gaps in the input, different output placement (reversed order)
    ioff, pos = [], 0
    for n in lengths:
        pos += 3
        ioff.append(pos)
        pos += n
    total_in = pos + 5
    ooff, pos = [0] * len(lengths), 0
    for i in reversed(range(len(lengths))):
        ooff[i] = pos
        pos += lengths[i] + 1
    src = np.zeros(total_in, np.complex128)
    for i, n in enumerate(lengths):
        src[ioff[i]:ioff[i] + n] = parts[i]
    v = UnevenBatch("f64", lengths, ioff, ooff)
    out = torch.zeros(pos, dtype=torch.complex128, device="cuda")
    v(torch.from_numpy(src).cuda(), out=out)
    assert v.status() == 0
    check_all(lengths, out.cpu().numpy(), parts, "f64", out_offsets=ooff)


def test_graph_replay():
    from fft_b200.device import DevicePlan, Graph, UnevenBatch
    lengths = [4096, 1009, 60, 65536, 10007]
    parts, flat = make_batch(lengths, 7, np.complex64)
    u = UnevenBatch("f32mixed", lengths)
    p = DevicePlan("c2c", "f32mixed", [1024], batch=8)
    x = torch.from_numpy(flat).cuda()
    y = torch.empty_like(x)
    a = torch.randn(8, 1024, dtype=torch.complex64, device="cuda")
    b = torch.empty_like(a)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        u(x, out=y, stream=s)  # first run on these buffers (before capture)
        p.c2c(a, out=b, stream=s)
    s.synchronize()
    y.zero_()
    b.zero_()
    with torch.cuda.stream(s):
        with Graph(s) as g:
            u(x, out=y, stream=s)
            p.c2c(a, out=b, stream=s)
        for _ in range(3):
            g.replay()
    s.synchronize()
    assert u.status() == 0
    check_all(lengths, y.cpu().numpy(), parts, "f32mixed")
    want = O.batch_fft(a.cpu().numpy().astype(np.complex128))
    assert rel_l2(b.cpu().numpy(), want) <= 1e-6


def test_bounded_wait_reports_timeout():
    # a dependency that never completes: every wait gives up after its poll
    # limit, the kernel returns, the status is a timeout, and the context
    # stays usable
    from fft_b200._lib import GOFFT_ETIMEOUT
    from fft_b200.device import UnevenBatch
    lengths = [65536, 65536, 128]
    parts, flat = make_batch(lengths, 9, np.complex64)
    u = UnevenBatch("f32mixed", lengths)
    u.set(1, 200)   # poll limit
    u.set(2, 1)     # hook: wait on work that never completes
    x = torch.from_numpy(flat).cuda()
    u(x)
    assert u.status() == GOFFT_ETIMEOUT
    u.set(2, 0)
    u.set(1, 1 << 24)
    y = u(x)
    assert u.status() == 0
    check_all(lengths, y.cpu().numpy(), parts, "f32mixed")


def test_timeout_drains_at_default_limit():
    # at the default poll limit, a dependency that never completes must cost
    # about one wait, not one wait per dependent tile: once a CTA gives up,
    # the others stop waiting and the kernel drains.  The hook makes every
    # phase after the first wait; in the many-tile batch those phases hold
    # several times more tiles than CTAs (each CTA would otherwise wait the
    # full limit on every one of its tiles in turn).
    import time
    from fft_b200._lib import GOFFT_ETIMEOUT
    from fft_b200.device import UnevenBatch

    def timed(lengths):
        parts, flat = make_batch(lengths, 11, np.complex64)
        u = UnevenBatch("f32mixed", lengths)
        u.set(0, 1)   # the persistent launch
        u.set(2, 1)   # hook: the phases after the first wait on work that never completes
        d = u.describe()
        x = torch.from_numpy(flat).cuda()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u(x)
        st = u.status()
        dt = time.perf_counter() - t0
        assert st == GOFFT_ETIMEOUT
        u.set(2, 0)
        y = u(x)
        assert u.status() == 0
        check_all(lengths, y.cpu().numpy(), parts, "f32mixed")
        return dt, sum(ph["tiles"] for ph in d["phase_list"][1:]), d["grid"]

    t_one, tiles_one, grid = timed([65536, 128])
    t_many, tiles_many, _ = timed([65536] * 160 + [128])
    assert tiles_one <= grid and tiles_many >= 4 * grid, (tiles_one, tiles_many, grid)
    assert t_many < 2.0 * t_one + 1.0, (t_one, t_many)
