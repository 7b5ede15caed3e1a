"""Rader transforms whose convolution runs in one CTA's shared memory
(rader_ip.cuh): forward and inverse against the oracle for linear and cyclic
convolutions, FP64 and the FP32 forms, in place and out of place, and the
integer tables that drive them (perm, iperm, conv length) bit-exact."""
import numpy as np
import pytest
import torch

from conftest import rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32mixed": 1e-6, "f32": 2e-6}
CDT = {"f64": torch.complex128, "f32mixed": torch.complex64, "f32": torch.complex64}

# (precision, prime): the 10007-point signals of the uneven batch
# (cl = 20580 = 4*3*5*7^3); cl = 7^5 = 16807; the longest that fits,
# cl = 27440 (219 KB of complex64); in FP64 a linear convolution of 8232 and
# cyclic ones of 8232 and 13720
CASES = [("f32mixed", 10007), ("f32", 10007), ("f32mixed", 7369), ("f32mixed", 13697),
         ("f64", 3923), ("f64", 8233), ("f64", 13721)]


@pytest.mark.parametrize("prec,p", CASES)
def test_rader_inplace_vs_oracle(prec, p):
    from fft_b200.device import DevicePlan
    B = 3
    d = DevicePlan("c2c", prec, [p], batch=B)
    ax = d.describe()["axes"][0]
    assert ax["engine"] == "rader" and ax["inplace"] == 1, ax
    info = O.rader_info(p)
    assert ax["cl"] == info["cl"] and ax["cyclic"] == int(info["cyclic"])
    g = rng(p)
    x = g.standard_normal((B, p)) + 1j * g.standard_normal((B, p))
    xt = torch.from_numpy(x).to(CDT[prec]).cuda()
    xd = xt.cpu().numpy().astype(np.complex128)
    for inverse in (False, True):
        y = d.c2c(xt, inverse=inverse).cpu().numpy()
        for b in range(B):
            want = (O.ifft if inverse else O.fft)(xd[b])
            assert rel_l2(y[b], want) <= TOL[prec], (prec, p, inverse, b)
    # in place
    z = xt.clone()
    d.c2c(z, out=z)
    assert rel_l2(z[1].cpu().numpy(), O.fft(xd[1])) <= TOL[prec]


@pytest.mark.parametrize("p", [10007, 13721])
def test_rader_inplace_tables(p):
    from fft_b200.device import DevicePlan
    d = DevicePlan("c2c", "f64" if p == 13721 else "f32mixed", [p])
    g, cl = d.table(3)
    info = O.rader_info(p)
    assert (g, cl) == (info["g"], info["cl"])
    np.testing.assert_array_equal(d.table(0), info["perm"])
    np.testing.assert_array_equal(d.table(1), info["iperm"])
