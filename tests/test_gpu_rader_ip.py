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

# (precision, prime): convolutions too long for one CTA, on a cluster of two
# CTAs each holding half: FP64 10007 (linear, cl = 20580 = 4*3*5*7^3, first
# radix 4), FP64 14851 (cyclic 14850 = 2*3^3*5^2*11, first radix 2), FP64
# 15361 (cyclic 15360 = 2^10*3*5, radices 8,8,4,4,3,5), FP32-mixed 14411
# (linear 29400 = 8*3*5^2*7^2, 235 KB of complex64)
PAIR_CASES = [("f64", 10007), ("f64", 14851), ("f64", 15361), ("f32mixed", 14411)]


@pytest.mark.parametrize("prec,p", CASES + PAIR_CASES)
def test_rader_inplace_vs_oracle(prec, p):
    from fft_b200.device import DevicePlan
    B = 3
    d = DevicePlan("c2c", prec, [p], batch=B)
    ax = d.describe()["axes"][0]
    assert ax["engine"] == "rader" and ax["inplace"] == 1, ax
    assert ax["inplace_ctas"] == (2 if (prec, p) in PAIR_CASES else 1), ax
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


def test_rader_pair_many_signals_strided():
    """FP64 10007 on CTA pairs over more signals than there are clusters
    (each cluster takes several), from a strided layout (the rows of a
    column-major block: element stride = the signal count)."""
    from fft_b200.device import DevicePlan
    p, B = 10007, 200
    g = rng(77)
    x = g.standard_normal((B, p)) + 1j * g.standard_normal((B, p))
    d = DevicePlan("c2c", "f64", [p], batch=B)
    assert d.describe()["axes"][0]["inplace_ctas"] == 2
    y = d.c2c(torch.from_numpy(x).cuda()).cpu().numpy()
    for b in (0, 73, 148, B - 1):
        assert rel_l2(y[b], O.fft(x[b])) <= TOL["f64"], b
    # FFTN over a (p, 3) array: the p-point axis has element stride 3
    z = g.standard_normal((p, 3)) + 1j * g.standard_normal((p, 3))
    n = DevicePlan("c2c", "f64", [p, 3])
    got = n.c2c(torch.from_numpy(z.reshape(1, -1)).cuda()).cpu().numpy().ravel()
    assert rel_l2(got, O.fftn(z, [p, 3])) <= TOL["f64"]
