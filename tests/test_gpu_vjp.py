"""Adjoint (VJP) kernels and the fused 2-D spectral filter: dot-product tests
of every transform's adjoint, gradients against the ones assembled from the
oracle's transforms, and central finite differences on the differentiation
workload (32 float32 512x512 images, a 512x257 Gaussian low-pass filter with
random phase)."""
import numpy as np
import pytest
import torch

from conftest import edge_weights, filter_case, filter_oracle, rdot, rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CDT = {"f64": torch.complex128, "f32mixed": torch.complex64, "f32": torch.complex64}
RDT = {"f64": torch.float64, "f32mixed": torch.float32, "f32": torch.float32}
# dot-product identities: rounding of one forward and one adjoint transform
DOT_TOL = {"f64": 1e-12, "f32mixed": 2e-6, "f32": 2e-6}
# gradients against the oracle's FP64 assembly (relative L2)
GRAD_TOL = {"f64": 1e-12, "f32mixed": 1e-6, "f32": 2e-6}


def crand(g, shape, dt):
    return torch.from_numpy(g.standard_normal(shape) + 1j * g.standard_normal(shape)).to(dt).cuda()


def rrand(g, shape, dt):
    return torch.from_numpy(g.standard_normal(shape)).to(dt).cuda()


def tdot(a, b):
    return rdot(a.cpu().numpy(), b.cpu().numpy())


@pytest.mark.parametrize("prec", ["f64", "f32mixed", "f32"])
@pytest.mark.parametrize("shape", [[1024], [1000], [1009], [10007], [262144], [64, 48], [5, 7, 9]])
def test_dot_c2c(prec, shape):
    from fft_b200.device import DevicePlan
    g = rng(21)
    B = 3
    N = int(np.prod(shape))
    p = DevicePlan("c2c", prec, shape, batch=B)
    for inverse in (False, True):
        x = crand(g, (B, N), CDT[prec])
        G = crand(g, (B, N), CDT[prec])
        lhs = tdot(p.c2c(x, inverse=inverse), G)
        rhs = tdot(x, p.vjp_c2c(G, inverse=inverse))
        scale = float(torch.linalg.norm(x.to(torch.complex128)) * torch.linalg.norm(G.to(torch.complex128)))
        scale *= np.sqrt(N) if not inverse else 1.0 / np.sqrt(N)
        assert abs(lhs - rhs) <= DOT_TOL[prec] * scale, (shape, inverse, lhs, rhs)


@pytest.mark.parametrize("prec", ["f64", "f32mixed", "f32"])
@pytest.mark.parametrize("shape", [[1024], [1001], [2], [1], [65536], [1 << 20], [64, 64], [30, 17], [1, 12], [9, 1]])
def test_dot_real(prec, shape):
    from fft_b200.device import DevicePlan
    g = rng(22)
    B = 2
    N = int(np.prod(shape))
    p = DevicePlan("r2c", prec, shape, batch=B)
    x = rrand(g, (B, N), RDT[prec])
    G = crand(g, (B, p.bins), CDT[prec])
    nx = float(torch.linalg.norm(x.double()))
    nG = float(torch.linalg.norm(G.to(torch.complex128)))
    # <RFFT x, G> = <x, RFFT^T G>
    lhs = tdot(p.r2c(x), G)
    rhs = tdot(x, p.vjp_r2c(G))
    assert abs(lhs - rhs) <= DOT_TOL[prec] * np.sqrt(N) * nx * nG, (shape, lhs, rhs)
    # <IRFFT G, y> = <G, IRFFT^T y>
    y = rrand(g, (B, N), RDT[prec])
    ny = float(torch.linalg.norm(y.double()))
    lhs = tdot(p.c2r(G), y)
    rhs = tdot(G, p.vjp_c2r(y))
    assert abs(lhs - rhs) <= DOT_TOL[prec] * nG * ny / np.sqrt(N) * 4, (shape, lhs, rhs)


@pytest.mark.parametrize("n", [1024, 1001, 16])
def test_vjp_real_vs_oracle(n):
    """The adjoints against the formulas evaluated with the oracle's
    transforms: RFFT^T(G) = N IRFFT(G / w), IRFFT^T(g) = (w / N) RFFT(g)."""
    from fft_b200.device import DevicePlan
    g = rng(23)
    p = DevicePlan("r2c", "f64", [n], batch=1)
    w = edge_weights(n)
    G = g.standard_normal(n // 2 + 1) + 1j * g.standard_normal(n // 2 + 1)
    got = p.vjp_r2c(torch.from_numpy(G[None]).cuda()).cpu().numpy()[0]
    assert rel_l2(got, n * O.irfft(G / w, n)) <= 1e-12
    y = g.standard_normal(n)
    got = p.vjp_c2r(torch.from_numpy(y[None]).cuda()).cpu().numpy()[0]
    assert rel_l2(got, w / n * O.rfft(y)) <= 1e-12
    q = DevicePlan("c2c", "f64", [n], batch=1)
    z = g.standard_normal(n) + 1j * g.standard_normal(n)
    got = q.vjp_c2c(torch.from_numpy(z[None]).cuda()).cpu().numpy()[0]
    assert rel_l2(got, n * O.ifft(z)) <= 1e-12
    got = q.vjp_c2c(torch.from_numpy(z[None]).cuda(), inverse=True).cpu().numpy()[0]
    assert rel_l2(got, O.fft(z) / n) <= 1e-12


def run_filter(prec, x, H, saved=True):
    from fft_b200.function import SpectralFilter2
    B, R, C = x.shape
    f = SpectralFilter2(prec, R, C, batch=B)
    xt = torch.from_numpy(x).to(RDT[prec]).cuda()
    Ht = torch.from_numpy(H).to(CDT[prec]).cuda()
    y = f.Forward(xt.reshape(B, R * C), Ht.reshape(-1), need_dh=saved)
    return f, xt, Ht, y


@pytest.fixture(scope="module")
def c5():
    x, H = filter_case()
    y, dx, dH = filter_oracle(x, H)
    return x, H, y, dx, dH


@pytest.mark.parametrize("prec", ["f64", "f32mixed", "f32"])
def test_filter2_workload_vs_oracle(prec, c5):
    x, H, y_o, dx_o, dH_o = c5
    B, R, C = x.shape
    f, xt, Ht, y = run_filter(prec, x, H)
    assert rel_l2(y.cpu().numpy().reshape(B, R, C), y_o) <= GRAD_TOL[prec]
    dx, dH = f.Backward(2 * y)
    assert rel_l2(dx.cpu().numpy().reshape(B, R, C), dx_o) <= GRAD_TOL[prec]
    assert rel_l2(dH.cpu().numpy().reshape(R, -1), dH_o) <= GRAD_TOL[prec]


# relative part of the finite-difference tolerance, and the unit roundoff
FD_RTOL = {"f64": 1e-6, "f32mixed": 2e-2, "f32": 2e-2}
FD_U = {"f64": 2.0 ** -53, "f32mixed": 2.0 ** -24, "f32": 2.0 ** -24}
# rounding floor of the central differences, in units of u L' / h (see fd_check)
FD_FLOOR = 16


def fd_check(f, xt, Ht, y, dx, dH, eps, rtol, u, seed=24, n_x=32, n_h=32):
    """Central differences of L = sum(y^2) against the analytic gradients on
    n_x coordinates of x and n_h of H (real or imaginary parts).

    L(+) - L(-) is evaluated as sum((y+ - y-) (y+ + y-)) in FP64 from the
    engine's outputs (images the step leaves alone are bitwise equal and
    cancel).  L is quadratic, so the central difference is exact for every
    step and what remains is rounding.  Tolerance per coordinate: the
    rounding floor of a difference quotient, FD_FLOOR u L' / h (u the unit
    roundoff, L' the part of L the step changes, h the step), plus
    rtol |gradient|.  The rounding of L(+) - L(-) was measured at up to
    4.7 u L' on this workload (FP64, x coordinate (3, 308, 366) of seed 24:
    2.07e-6 against a gradient of 0.038 at h = 2e-6, L' = 7934), so the floor
    is 16 u L' / h, about three times that.  In FP32 the floor exceeds the x
    gradients of 512 x 512 images (L' is about 6.6e4 per image for a step of
    2e-3): there the check is a bound, and the callers add closeness checks on the coordinates whose
    gradients stand well above it.  The difference at 2 eps is evaluated as
    well and held to the same bound (the gradient must not depend on the
    step)."""
    B = xt.shape[0]
    R, K = Ht.shape
    C = xt.shape[2]
    yy = y.double().reshape(B, -1) ** 2
    L_img = [float(v) for v in yy.sum(dim=1)]
    L_all = float(sum(L_img))

    def dloss(xp, xm, Hp, Hm):
        yp = f.plan.filter2(xp.reshape(B, -1), Hp.reshape(-1)).double()
        ym = f.plan.filter2(xm.reshape(B, -1), Hm.reshape(-1)).double()
        return float(torch.sum((yp - ym) * (yp + ym)))

    def fd_x(b, i, j, e):
        xp, xm = xt.clone(), xt.clone()
        xp[b, i, j] += e
        xm[b, i, j] -= e
        step = float(xp[b, i, j].double() - xm[b, i, j].double())  # as stored
        return dloss(xp, xm, Ht, Ht) / step

    def fd_h(r, k, unit, e):
        Hp, Hm = Ht.clone(), Ht.clone()
        Hp[r, k] += e * unit
        Hm[r, k] -= e * unit
        dv = (Hp[r, k] - Hm[r, k]).to(torch.complex128)
        step = float(dv.real if unit == 1.0 else dv.imag)
        return dloss(xt, xt, Hp, Hm) / step

    g = rng(seed)
    checked = []
    for _ in range(n_x):
        b, i, j = (int(v) for v in (g.integers(0, B), g.integers(0, R), g.integers(0, C)))
        a1, a2 = fd_x(b, i, j, eps), fd_x(b, i, j, 2 * eps)
        want = float(dx[b, i, j])
        assert abs(a1 - want) <= FD_FLOOR * u * L_img[b] / (2 * eps) + rtol * abs(want), ("x", b, i, j, a1, want)
        assert abs(a2 - want) <= FD_FLOOR * u * L_img[b] / (4 * eps) + rtol * abs(want), ("x2", b, i, j, a2, want)
        checked.append((abs(want), abs(a1 - want) / (abs(want) + 1e-300)))
    for q in range(n_h):
        r, k = int(g.integers(0, R)), int(g.integers(0, K))
        unit = 1.0 if q % 2 == 0 else 1j
        a1, a2 = fd_h(r, k, unit, eps), fd_h(r, k, unit, 2 * eps)
        want = float(dH[r, k].real if unit == 1.0 else dH[r, k].imag)
        assert abs(a1 - want) <= FD_FLOOR * u * L_all / (2 * eps) + rtol * abs(want), ("H", r, k, unit, a1, want)
        assert abs(a2 - want) <= FD_FLOOR * u * L_all / (4 * eps) + rtol * abs(want), ("H2", r, k, unit, a2, want)
        checked.append((abs(want), abs(a1 - want) / (abs(want) + 1e-300)))
    return checked


@pytest.mark.parametrize("prec,eps", [("f64", 1e-6), ("f32mixed", 1e-3), ("f32", 1e-3)])
def test_filter2_finite_differences(prec, eps, c5):
    """Central differences on the differentiation workload, 64 random
    coordinates (32 of x, 32 of H); eps 1e-6 in FP64, 1e-3 in FP32."""
    x, H, y_o, dx_o, dH_o = c5
    B, R, C = x.shape
    f, xt, Ht, y = run_filter(prec, x, H)
    dx, dH = f.Backward(2 * y)
    checked = fd_check(f, xt, Ht.reshape(R, -1), y, dx.cpu().numpy().reshape(B, R, C),
                       dH.cpu().numpy().reshape(R, -1), eps, FD_RTOL[prec], FD_U[prec])
    # coordinates whose gradients stand well above the rounding floor agree closely
    if prec == "f64":
        big = [e for m, e in checked if m > 1e-3]
        assert len(big) >= 32 and max(big) <= 1e-4
    else:
        big = [e for m, e in checked if m > 0.5]
        assert len(big) >= 2 and max(big) <= 2e-2


@pytest.mark.parametrize("prec", ["f32mixed", "f32"])
def test_filter2_finite_differences_small_fp32(prec):
    """FP32 central differences (eps 1e-3) where the rounding floor sits
    below the gradients: 2 centred 16 x 16 images, loss of order 10."""
    x, H = filter_case(batch=2, rows=16, cols=16, seed_x=6)
    x = x - np.float32(0.5)
    f, xt, Ht, y = run_filter(prec, x, H)
    dx, dH = f.Backward(2 * y)
    checked = fd_check(f, xt, Ht.reshape(16, -1), y, dx.cpu().numpy().reshape(x.shape),
                       dH.cpu().numpy().reshape(16, -1), 1e-3, FD_RTOL[prec], FD_U[prec])
    big = [e for m, e in checked if m > 0.05]
    assert len(big) >= 24 and float(np.median(big)) <= 1e-2


@pytest.mark.parametrize("prec", ["f64", "f32mixed"])
@pytest.mark.parametrize("B,R,C", [(3, 1009, 48), (2, 1, 20), (2, 12, 1), (2, 40, 31), (5, 64, 64)])
def test_filter2_shapes(prec, B, R, C):
    """Prime and odd image sides (the column pass outside one CTA, odd real
    rows), a single row and a single column."""
    g = rng(25)
    x = g.random((B, R, C)).astype(np.float32)
    K = C // 2 + 1
    H = (g.standard_normal((R, K)) + 1j * g.standard_normal((R, K))).astype(np.complex64)
    up = g.standard_normal((B, R, C))
    y_o, dx_o, dH_o = filter_oracle(x, H, g=up)
    f, xt, Ht, y = run_filter(prec, x, H)
    assert rel_l2(y.cpu().numpy().reshape(B, R, C), y_o) <= GRAD_TOL[prec]
    dx, dH = f.Backward(torch.from_numpy(up.reshape(B, -1)).to(RDT[prec]).cuda())
    assert rel_l2(dx.cpu().numpy().reshape(B, R, C), dx_o) <= GRAD_TOL[prec]
    assert rel_l2(dH.cpu().numpy().reshape(R, K), dH_o) <= GRAD_TOL[prec]


def test_autograd_bridge():
    """torch.autograd through the Function interface gives the engine's own
    gradients; torch.fft's autograd of the same loss agrees (a second,
    independent derivation)."""
    from fft_b200.function import RFFT, SpectralFilter2, apply
    x, H = filter_case(batch=4, rows=64, cols=48)
    B, R, C = x.shape
    xt = torch.from_numpy(x).double().cuda().reshape(B, R * C).requires_grad_(True)
    Ht = torch.from_numpy(H).to(torch.complex128).cuda().reshape(-1).requires_grad_(True)
    f = SpectralFilter2("f64", R, C, batch=B)
    y = apply(f, xt, Ht)
    (y ** 2).sum().backward()
    xr = xt.detach().clone().reshape(B, R, C).requires_grad_(True)
    Hr = Ht.detach().clone().reshape(R, -1).requires_grad_(True)
    yr = torch.fft.irfft2(Hr * torch.fft.rfft2(xr), s=(R, C))
    (yr ** 2).sum().backward()
    assert rel_l2(xt.grad.cpu().numpy().ravel(), xr.grad.cpu().numpy().ravel()) <= 1e-12
    assert rel_l2(Ht.grad.cpu().numpy().ravel(), Hr.grad.cpu().numpy().ravel()) <= 1e-12
    # a transform alone: sum |RFFT(x)|^2 weighted
    r = RFFT("f64", [256], batch=2)
    a = torch.randn(2, 256, dtype=torch.float64, device="cuda", requires_grad=True)
    S = apply(r, a)
    (S.abs() ** 2).sum().backward()
    a2 = a.detach().clone().requires_grad_(True)
    (torch.fft.rfft(a2).abs() ** 2).sum().backward()
    assert rel_l2(a.grad.cpu().numpy(), a2.grad.cpu().numpy()) <= 1e-12


def test_filter2_without_dh():
    x, H = filter_case(batch=2, rows=32, cols=32)
    y_o, dx_o, _ = filter_oracle(x, H)
    f, xt, Ht, y = run_filter("f64", x, H, saved=False)
    dx, dH = f.Backward(2 * y)
    assert dH is None
    assert rel_l2(dx.cpu().numpy().reshape(x.shape), dx_o) <= 1e-12
