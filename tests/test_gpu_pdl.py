"""Programmatic dependent launch of the line kernels (gofft_set_dependent_launch):
in every mode the chained passes of a 2-D real round trip, a four-step 1-D
batch and an uneven batch give bit-identical results (the same kernels run;
only when their CTAs may be scheduled changes), and match the oracle."""
import numpy as np
import pytest
import torch

from conftest import rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def pdl_mode():
    from fft_b200 import tune
    yield tune.set_dependent_launch
    tune.set_dependent_launch(0)


def _round_trip(prec, mode, x, set_mode):
    from fft_b200.device import DevicePlan
    set_mode(mode)
    p = DevicePlan("r2c", prec, [1024, 1024], batch=x.shape[0])
    X = p.r2c(x)
    back = p.c2r(X)
    torch.cuda.synchronize()
    return X.cpu().numpy(), back.cpu().numpy()


@pytest.mark.parametrize("prec", ["f64", "f32mixed"])
def test_pdl_round_trip_identical(prec, pdl_mode):
    B = 6
    rdt = torch.float64 if prec == "f64" else torch.float32
    x = torch.from_numpy(rng(51).standard_normal((B, 1024 * 1024))).to(rdt).cuda()
    X0, b0 = _round_trip(prec, 0, x, pdl_mode)
    for mode in (1, 2):
        X, b = _round_trip(prec, mode, x, pdl_mode)
        np.testing.assert_array_equal(X, X0)
        np.testing.assert_array_equal(b, b0)
    tol = 1e-12 if prec == "f64" else 1e-6
    want = O.rfft2(x[B - 1].double().cpu().numpy(), 1024, 1024)
    assert rel_l2(X0[B - 1], want) <= tol
    assert rel_l2(b0, x.cpu().numpy()) <= tol


def test_pdl_fourstep_and_uneven_identical(pdl_mode):
    from fft_b200.device import DevicePlan, UnevenBatch
    g = rng(52)
    n, B = 65536, 200
    x = torch.from_numpy(g.standard_normal((B, n)) + 1j * g.standard_normal((B, n))).cuda()
    lens = [int(v) for v in g.choice([60, 1000, 1009, 4096, 10007, 65536], 64)]
    flat = (g.uniform(-1, 1, sum(lens)) + 1j * g.uniform(-1, 1, sum(lens))).astype(np.complex64)
    xf = torch.from_numpy(flat).cuda()
    outs = []
    for mode in (0, 1, 2):
        pdl_mode(mode)
        p = DevicePlan("c2c", "f64", [n], batch=B)
        y = p.c2c(x)
        z = p.c2c(y, inverse=True)
        u = UnevenBatch("f32mixed", lens)
        u.set(0, 0)
        w = u(xf)
        torch.cuda.synchronize()
        assert u.status() == 0
        outs.append((y.cpu().numpy(), z.cpu().numpy(), w.cpu().numpy()))
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            np.testing.assert_array_equal(a, b)
    y0 = outs[0][0]
    assert rel_l2(y0[B - 1], O.fft(x[B - 1].cpu().numpy())) <= 1e-12
    assert rel_l2(outs[0][1], x.cpu().numpy()) <= 1e-12
    off = sum(lens[:-1])
    assert rel_l2(outs[0][2][off:], O.fft(flat[off:].astype(np.complex128))) <= 1e-6
