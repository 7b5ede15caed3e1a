"""The TMA-fed persistent line kernel (k_pipe): the passes of the 2-D real
round trip, batched complex rows and complex 2-D columns give the same
results with it as with the one-tile-per-CTA kernels, and match the oracle.
Each case checks that the pipelined kernel really ran (its launches are
named .../pipe/... in the engine's timing report) and that none of its
bounded waits gave up (gofft_pipeline_status)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# pipelined against the other kernels: the same stages and tables, so they
# differ at most by the compiler's choice of fused multiply-adds
SAME = {"f64": 2e-15, "f32mixed": 2e-7}
ORACLE = {"f64": 1e-12, "f32mixed": 1e-6}


def _run(fn, pipe):
    from fft_b200 import _lib, tune
    tune.set_tma_pipeline(pipe)
    _lib.timing_enable(True)
    _lib.timing_report()
    try:
        out = fn()
        torch.cuda.synchronize()
        kernels = [r["kernel"] for r in _lib.timing_report()]
    finally:
        _lib.timing_enable(False)
        tune.set_tma_pipeline(False)
    tune.pipeline_status()
    return out, kernels


def _both(fn, want_pipe_ops):
    ref, k_off = _run(fn, False)
    got, k_on = _run(fn, True)
    assert not any("/pipe/" in k for k in k_off)
    for op in want_pipe_ops:
        assert any(k.startswith(op + "/") and "/pipe/" in k for k in k_on), (op, k_on)
    return ref, got


@pytest.fixture
def schedule():
    from fft_b200._lib import lib
    set_to = []

    def apply(prec, n, v):
        lib().gofft_set_schedule(prec, n, v)
        set_to.append((prec, n))
    yield apply
    for prec, n in set_to:
        lib().gofft_set_schedule(prec, n, 0)


@pytest.mark.parametrize("prec,variant", [("f64", 0), ("f64", 1), ("f32mixed", 0)])
def test_pipe_rfft2_1024(prec, variant, schedule):
    """Rows (packed R2C / C2R, 512-point), columns (1024-point): FP64 columns
    by 2-D tensor copies, FP32 columns (4104-byte rows) by element copies."""
    from fft_b200.device import DevicePlan
    from fft_b200._lib import GOFFT_F64, GOFFT_F32MIXED
    schedule(GOFFT_F64 if prec == "f64" else GOFFT_F32MIXED, 512, variant)
    # every L2 block (two per plan at least) needs two tiles per SM for the
    # pipelined kernel: 6 FP64 images make blocks of 3, 8 FP32 images of 4
    B = 6 if prec == "f64" else 8
    rdt = torch.float64 if prec == "f64" else torch.float32
    x = rng(31).standard_normal((B, 1024 * 1024))
    xt = torch.from_numpy(x).to(rdt).cuda()
    p = DevicePlan("r2c", prec, [1024, 1024], batch=B)
    ref, got = _both(lambda: p.r2c(xt), ["r2c_packed", "c2c"])
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= SAME[prec]
    for b in (0, B - 1):
        want = O.rfft2(xt[b].double().cpu().numpy(), 1024, 1024)
        assert rel_l2(got[b].cpu().numpy(), want) <= ORACLE[prec]
    back_ref, back = _both(lambda: p.c2r(got), ["c2r_packed", "c2c"])
    assert rel_l2(back.cpu().numpy(), back_ref.cpu().numpy()) <= SAME[prec]
    assert rel_l2(back.cpu().numpy(), xt.cpu().numpy()) <= ORACLE[prec]


@pytest.mark.parametrize("prec", ["f64", "f32mixed"])
def test_pipe_row_tail(prec):
    """1001 rows per image: the last row tile is partial (FP32: its bins are
    not a multiple of 16 bytes, so that tile falls back to element copies)."""
    from fft_b200.device import DevicePlan
    B, R, C = 6, 1001, 1024
    rdt = torch.float64 if prec == "f64" else torch.float32
    x = rng(32).standard_normal((B, R * C))
    xt = torch.from_numpy(x).to(rdt).cuda()
    p = DevicePlan("r2c", prec, [R, C], batch=B)
    ref, got = _both(lambda: p.r2c(xt), ["r2c_packed"])
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= SAME[prec]
    want = O.rfft2(xt[B - 1].double().cpu().numpy(), R, C)
    assert rel_l2(got[B - 1].cpu().numpy(), want) <= ORACLE[prec]
    back_ref, back = _both(lambda: p.c2r(got), ["c2r_packed"])
    assert rel_l2(back.cpu().numpy(), back_ref.cpu().numpy()) <= SAME[prec]
    assert rel_l2(back.cpu().numpy(), xt.cpu().numpy()) <= ORACLE[prec]


def test_pipe_complex_rows_and_columns():
    """Batched 1024-point complex rows (bulk row copies) and the column pass
    of a batch of two 1024 x 1024 complex 2-D transforms (tensor copies)."""
    from fft_b200.device import DevicePlan
    g = rng(33)
    x = g.standard_normal((2048, 1024)) + 1j * g.standard_normal((2048, 1024))
    xt = torch.from_numpy(x).cuda()
    p = DevicePlan("c2c", "f64", [1024], batch=2048)
    for inverse in (False, True):
        ref, got = _both(lambda: p.c2c(xt, inverse=inverse), ["c2c"])
        assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= SAME["f64"]
        want = (O.ifft if inverse else O.fft)(x[5])
        assert rel_l2(got[5].cpu().numpy(), want) <= ORACLE["f64"]
    y = g.standard_normal((2, 1024 * 1024)) + 1j * g.standard_normal((2, 1024 * 1024))
    yt = torch.from_numpy(y).cuda()
    q = DevicePlan("c2c", "f64", [1024, 1024], batch=2)
    ref, got = _both(lambda: q.c2c(yt), ["c2c"])
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= SAME["f64"]
    want = O.fftn(y[1], [1024, 1024])
    assert rel_l2(got[1].cpu().numpy(), want) <= ORACLE["f64"]


def test_pipe_adjoints():
    """The real adjoints run the packed rows with the edge-bin weights."""
    from fft_b200.device import DevicePlan
    B = 6
    g = rng(34)
    p = DevicePlan("r2c", "f64", [1024, 1024], batch=B)
    G = torch.from_numpy(g.standard_normal((B, 1024 * 513)) + 1j * g.standard_normal((B, 1024 * 513))).cuda()
    ref, got = _both(lambda: p.vjp_r2c(G), ["c2r_packed"])
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= SAME["f64"]
    xr = torch.from_numpy(g.standard_normal((B, 1024 * 1024))).cuda()
    ref, got = _both(lambda: p.vjp_c2r(xr), ["r2c_packed"])
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= SAME["f64"]
