"""The autotuner and the radix-8 / radix-32 schedule variants: tuned and varied plans
still match the oracle (settings are process-wide, so every test here puts
the defaults back)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32mixed": 1e-6, "f32": 1e-6}
PREC = {"f64": 0, "f32": 1, "f32mixed": 2}


@pytest.fixture(autouse=True)
def defaults():
    from fft_b200 import tune
    tune.forget_wisdom()
    yield
    tune.forget_wisdom()


@pytest.mark.parametrize("var", [1, 2])
@pytest.mark.parametrize("prec", ["f64", "f32mixed", "f32"])
@pytest.mark.parametrize("n", [8, 64, 128, 256, 512, 1024, 2048, 4096, 360, 1000, 1009, 10007, 65536])
def test_variant_c2c(var, prec, n):
    from fft_b200._lib import lib
    from fft_b200.device import DevicePlan
    for m in {n, 1008, 256}:
        lib().gofft_set_schedule(PREC[prec], m, var)
    B = 5
    g = rng(n)
    x = g.standard_normal((B, n)) + 1j * g.standard_normal((B, n))
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    p = DevicePlan("c2c", prec, [n], batch=B)
    xt = torch.from_numpy(x).to(cdt).cuda()
    assert rel_l2(p.c2c(xt).cpu().numpy(), O.batch_fft(x)) <= TOL[prec]
    assert rel_l2(p.c2c(xt, inverse=True).cpu().numpy(), O.batch_fft(x, inverse=True)) <= TOL[prec]


@pytest.mark.parametrize("var", [1, 2])
@pytest.mark.parametrize("prec", ["f64", "f32mixed", "f32"])
@pytest.mark.parametrize("shape", [[1024, 1024], [512, 512], [256, 512], [64, 2048], [30, 1000]])
def test_variant_rfft2(var, prec, shape):
    from fft_b200._lib import lib
    from fft_b200.device import DevicePlan
    R, C = shape
    for m in {R, C // 2}:
        lib().gofft_set_schedule(PREC[prec], m, var)
    B = 3
    x = rng(R + C).standard_normal((B, R, C))
    rdt = torch.float64 if prec == "f64" else torch.float32
    p = DevicePlan("r2c", prec, shape, batch=B)
    X = p.r2c(torch.from_numpy(x.reshape(B, -1)).to(rdt).cuda())
    want = np.stack([O.rfft2(x[b], R, C) for b in range(B)])
    assert rel_l2(X.cpu().numpy(), want) <= TOL[prec]
    back = p.c2r(X).cpu().numpy().reshape(B, R, C)
    assert rel_l2(back, np.stack([O.irfft2(want[b], R, C).reshape(R, C) for b in range(B)])) <= TOL[prec]


def test_autotune_rfft2_keeps_parity():
    from fft_b200 import tune
    from fft_b200.device import DevicePlan
    w = tune.autotune("r2c", "f64", [256, 256], batch=8)
    assert w["gofft_wisdom"] == 1
    x = rng(5).standard_normal((8, 256, 256))
    p = DevicePlan("r2c", "f64", [256, 256], batch=8)
    X = p.r2c(torch.from_numpy(x.reshape(8, -1)).cuda()).cpu().numpy()
    assert rel_l2(X, np.stack([O.rfft2(x[b], 256, 256) for b in range(8)])) <= 1e-12
    # exported wisdom reproduces the same settings in a clean state
    text = tune.export_wisdom()
    tune.forget_wisdom()
    tune.import_wisdom(text)
    assert tune.export_wisdom() == text


def test_autotune_c2c_and_uneven():
    from fft_b200 import tune
    from fft_b200.device import DevicePlan, UnevenBatch
    tune.autotune("c2c", "f32mixed", [4096], batch=64)
    x = rng(6).standard_normal((64, 4096)) + 1j * rng(7).standard_normal((64, 4096))
    p = DevicePlan("c2c", "f32mixed", [4096], batch=64)
    y = p.c2c(torch.from_numpy(x).to(torch.complex64).cuda()).cpu().numpy()
    assert rel_l2(y, O.batch_fft(x)) <= 1e-6
    lengths = [60, 128, 360, 1000, 1009, 4096, 10007, 65536] * 3
    tune.autotune_uneven("f32mixed", lengths)
    parts = [rng(n).standard_normal(n) + 1j * rng(n + 1).standard_normal(n) for n in lengths]
    flat = np.concatenate(parts).astype(np.complex64)
    u = UnevenBatch("f32mixed", lengths)
    got = u(torch.from_numpy(flat).cuda()).cpu().numpy()
    assert u.status() == 0
    off = 0
    for part in parts:
        assert rel_l2(got[off:off + part.size], O.fft(part)) <= 1e-6
        off += part.size


def test_uneven_caps_variant2():
    """Uneven batches run every class in the persistent kernel's 16-element
    registers: a radix-32 setting for one of their lengths is capped, not
    run wrong."""
    from fft_b200._lib import lib
    from fft_b200.device import UnevenBatch
    lengths = [1024, 512, 4096, 1024, 60]
    for n in set(lengths):
        lib().gofft_set_schedule(PREC["f32mixed"], n, 2)
    parts = [rng(n).standard_normal(n) + 1j * rng(n + 3).standard_normal(n) for n in lengths]
    u = UnevenBatch("f32mixed", lengths)
    got = u(torch.from_numpy(np.concatenate(parts).astype(np.complex64)).cuda()).cpu().numpy()
    assert u.status() == 0
    off = 0
    for part in parts:
        assert rel_l2(got[off:off + part.size], O.fft(part)) <= 1e-6
        off += part.size
