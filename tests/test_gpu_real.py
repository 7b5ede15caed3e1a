"""Real and multi-dimensional transforms on the B200 against the oracle."""
import numpy as np
import pytest
import torch

from conftest import rel_l2, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12
F32_TOL = 1e-6

REAL_N = [1, 2, 3, 4, 5, 6, 7, 8, 9, 12, 15, 16, 17, 31, 32, 100, 128, 1000, 1024, 2048, 2018, 4096, 1009,
          131072, 20014]


@pytest.mark.parametrize("n", REAL_N)
def test_rfft_irfft_f64(n):
    from fft_b200 import gofft as G
    x = rng(n).standard_normal(n)
    X = G.RFFT(x)
    assert X.size == n // 2 + 1
    assert rel_l2(X, O.rfft(x)) <= F64_TOL
    back = G.IRFFT(X, n)
    assert rel_l2(back, O.irfft(X, n)) <= F64_TOL
    assert np.max(np.abs(back - x)) < 1e-9
    p = G.NewRealPlan(n)
    d = p.RFFT(np.zeros(n // 2 + 1, complex), x)
    assert rel_l2(d, O.rfft(x)) <= F64_TOL


@pytest.mark.parametrize("prec", ["f64", "f32mixed"])
@pytest.mark.parametrize("n", [1024, 1001, 262144, 12])
def test_batched_rank1_real_device(prec, n):
    """Batched 1-D R2C/C2R device plans: bins at n/2+1 per transform, reals
    at n (each side at its own distance), and a short spectrum (nbins)."""
    from fft_b200.device import DevicePlan
    B = 5
    g = rng(n + 7)
    x = g.standard_normal((B, n))
    p = DevicePlan("r2c", prec, [n], batch=B)
    rdt = torch.float64 if prec == "f64" else torch.float32
    tol = F64_TOL if prec == "f64" else F32_TOL
    X = p.r2c(torch.from_numpy(x).to(rdt).cuda())
    want = np.stack([O.rfft(r) for r in x])
    assert rel_l2(X.cpu().numpy(), want) <= tol
    back = p.c2r(X).cpu().numpy()
    assert rel_l2(back, np.stack([O.irfft(s, n) for s in want])) <= tol
    k = n // 4 + 1
    short = X.clone()
    short[:, k:] = 1e3  # bins past nbins are not read
    got = p.c2r(short, nbins=k).cpu().numpy()
    assert rel_l2(got, np.stack([O.irfft(s[:k], n) for s in want])) <= tol


def test_irfft_short_and_hermitian():
    # rfft_test.go:105-124, 190-198
    from fft_b200 import gofft as G
    half = np.array([3, 1 - 2j, -0.5 + 0.4j, 2])
    full = np.concatenate([half, np.conj(half[1:3][::-1])])
    assert np.max(np.abs(G.IRFFT(half, 6) - np.real(O.ifft(full)))) < 1e-9
    a = G.IRFFT(np.array([2 + 0j]), 4)
    b = G.IRFFT(np.array([2 + 0j, 0, 0]), 4)
    assert np.max(np.abs(a - b)) < 1e-12
    for n in [8, 9, 1024]:
        spec = rng(n).standard_normal(n // 2 + 1) + 1j * rng(n + 1).standard_normal(n // 2 + 1)
        for k in [1, 2, n // 4 + 1, n // 2 + 1]:
            assert rel_l2(G.IRFFT(spec[:k], n), O.irfft(spec[:k], n)) <= F64_TOL


@pytest.mark.parametrize("shape", [(4, 6), (3, 5), (2, 8), (5, 4), (1, 1), (7, 3), (1, 6), (6, 1), (33, 17),
                                   (1024, 1024), (512, 512), (9, 2018)])
def test_rfft2_irfft2_f64(shape):
    from fft_b200 import gofft as G
    r, c = shape
    x = rng(r * 1000 + c).standard_normal(r * c)
    X = G.RFFT2(x, shape)
    assert rel_l2(X, O.rfft2(x, r, c)) <= F64_TOL
    back = G.IRFFT2(X, shape)
    assert rel_l2(back, O.irfft2(X, r, c)) <= F64_TOL
    assert np.max(np.abs(back - x)) < 1e-9
    short = X[:-1]
    assert rel_l2(G.IRFFT2(short, shape), O.irfft2(short, r, c)) <= F64_TOL


@pytest.mark.parametrize("shape", [[2, 2], [3, 4], [4, 3], [1, 5], [5, 1], [2, 3, 4], [3, 1, 2], [2, 2, 2, 2],
                                   [6, 5], [64, 64, 64], [17, 1009], [3, 65536]])
def test_fftn_f64(shape):
    from fft_b200 import gofft as G
    n = int(np.prod(shape))
    g = rng(n)
    x = g.standard_normal(n) + 1j * g.standard_normal(n)
    X = G.FFTN(x, shape)
    assert rel_l2(X, O.fftn(x, shape)) <= F64_TOL
    back = G.IFFTN(X, shape)
    assert rel_l2(back, O.ifftn(X, shape)) <= F64_TOL
    if len(shape) == 2:
        assert rel_l2(G.FFT2(x, shape), X) <= F64_TOL
        assert rel_l2(G.IFFT2(X, shape), back) <= F64_TOL


def test_batched_rfft2_config2_shape():
    # RFFT2 then IRFFT2 of 1024x1024 float64 images, batched on device
    from fft_b200.device import DevicePlan
    B = 3
    x = rng(1).standard_normal((B, 1024, 1024))
    p = DevicePlan("r2c", "f64", [1024, 1024], batch=B)
    X = p.r2c(torch.from_numpy(x).cuda().reshape(B, -1))
    got = X.cpu().numpy().reshape(B, 1024, 513)
    for b in range(B):
        assert rel_l2(got[b].ravel(), O.rfft2(x[b], 1024, 1024)) <= F64_TOL
    back = p.c2r(X).cpu().numpy().reshape(B, 1024, 1024)
    assert np.max(np.abs(back - x)) < 1e-12


@pytest.mark.parametrize("prec", ["f64", "f32mixed"])
@pytest.mark.parametrize("shape,batch", [((1000, 64), 3), ((6, 720), 5), ((24, 512), 7), ((10, 30), 9),
                                         ((1024, 1024), 3), ((5, 8), 11)])
def test_rfft2_tiled_intermediate(prec, shape, batch):
    """Batched FP64 rank-2 real transforms keep the row-to-column intermediate
    in groups of four column-lines (the FP32 forms keep the image layout);
    image boundaries fall inside groups (rc not a multiple of 4), rows need
    not divide by the lines per CTA, and row lengths without a compiled
    kernel (720 = 2 x 360) take the run-time kernel.  Each image must match
    the oracle and invert to the input."""
    from fft_b200.device import DevicePlan
    R, C = shape
    K = C // 2 + 1
    tol = F64_TOL if prec == "f64" else F32_TOL
    g = rng(R * 7 + C + batch)
    x = g.standard_normal((batch, R, C))
    dt = np.float64 if prec == "f64" else np.float32
    p = DevicePlan("r2c", prec, [R, C], batch=batch)
    X = p.r2c(torch.from_numpy(x.astype(dt)).cuda().reshape(batch, -1))
    got = X.cpu().numpy().reshape(batch, R * K)
    for b in range(batch):
        assert rel_l2(got[b], O.rfft2(x[b], R, C)) <= tol
    back = p.c2r(X).cpu().numpy().reshape(batch, R, C)
    for b in range(batch):
        assert rel_l2(back[b], x[b]) <= (1e-13 if prec == "f64" else 2 * F32_TOL)


@pytest.mark.parametrize("pinned", [True, False])
def test_batched_rfft2_host_pipeline(pinned):
    # host-buffer RFFT2/IRFFT2 of a batch spanning several blocks on both
    # lanes (copies, transforms and copies back overlapped per block) must
    # give the device-buffer results
    from fft_b200.device import DevicePlan
    B = 8
    x = rng(9).standard_normal((B, 1024 * 1024))
    p = DevicePlan("r2c", "f64", [1024, 1024], batch=B)
    dev = p.r2c(torch.from_numpy(x).cuda())
    dev_back = p.c2r(dev).cpu().numpy()
    dev = dev.cpu().numpy()
    hx = torch.from_numpy(x)
    hs = torch.zeros((B, 1024 * 513), dtype=torch.complex128)
    hb = torch.zeros((B, 1024 * 1024), dtype=torch.float64)
    if pinned:
        hx, hs, hb = hx.pin_memory(), hs.pin_memory(), hb.pin_memory()
    for _ in range(2):
        p.r2c_host(hx.data_ptr(), hs.data_ptr())
        assert rel_l2(hs.numpy(), dev) <= 1e-15
        p.c2r_host(hs.data_ptr(), hb.data_ptr())
        assert rel_l2(hb.numpy(), dev_back) <= 1e-15
    assert rel_l2(hs.numpy()[B - 1], O.rfft2(x[B - 1].reshape(1024, 1024), 1024, 1024)) <= F64_TOL


@pytest.fixture
def small_l2_blocks():
    """A 1 MiB L2 block budget for the plans a test creates (restored after)."""
    from fft_b200 import tune
    tune.set_l2_block_bytes(1 << 20)
    yield 1 << 20
    tune.set_l2_block_bytes(0)


@pytest.mark.parametrize("pinned", [True, False])
def test_host_pipeline_one_image_blocks(pinned, small_l2_blocks):
    """A plan whose L2 block holds one image (each 256x256 float64 spectrum,
    526 KB, is more than half the 1 MiB budget): the host-buffer calls must not
    form blocks larger than a lane's workspace.  They take the serial path and
    match the device-buffer results exactly and the oracle at 1e-12."""
    from fft_b200.device import DevicePlan
    B, R, C = 6, 256, 256
    K = C // 2 + 1
    p = DevicePlan("r2c", "f64", [R, C], batch=B)
    assert p.describe()["chunk"] == 1
    x = rng(21).standard_normal((B, R * C))
    dev = p.r2c(torch.from_numpy(x).cuda())
    dev_back = p.c2r(dev).cpu().numpy()
    dev = dev.cpu().numpy()
    hx = torch.from_numpy(x)
    hs = torch.zeros((B, R * K), dtype=torch.complex128)
    hb = torch.zeros((B, R * C), dtype=torch.float64)
    if pinned:
        hx, hs, hb = hx.pin_memory(), hs.pin_memory(), hb.pin_memory()
    for _ in range(2):
        p.r2c_host(hx.data_ptr(), hs.data_ptr())
        assert np.array_equal(hs.numpy(), dev)
        p.c2r_host(hs.data_ptr(), hb.data_ptr())
        assert np.array_equal(hb.numpy(), dev_back)
    for b in range(B):
        assert rel_l2(hs.numpy()[b], O.rfft2(x[b].reshape(R, C), R, C)) <= F64_TOL
        assert np.max(np.abs(hb.numpy()[b] - x[b])) < 1e-12


@pytest.mark.parametrize("prec", ["f32", "f32mixed"])
def test_rfft2_fp32_forms(prec):
    from fft_b200.device import DevicePlan
    B, R, C = 4, 512, 512
    x = rng(4).uniform(0, 1, (B, R, C)).astype(np.float32)
    p = DevicePlan("r2c", prec, [R, C], batch=B)
    X = p.r2c(torch.from_numpy(x).cuda().reshape(B, -1)).cpu().numpy().reshape(B, -1)
    for b in range(B):
        assert rel_l2(X[b], O.rfft2(x[b].astype(np.float64), R, C)) <= F32_TOL
    back = p.c2r(torch.from_numpy(X).cuda()).cpu().numpy().reshape(B, R, C)
    assert rel_l2(back, x) <= 2 * F32_TOL


@pytest.mark.parametrize("prec", ["f32", "f32mixed"])
def test_fftn_3d_fp32(prec):
    from fft_b200.device import DevicePlan
    s = [64, 64, 64]
    g = rng(3)
    x = ((g.standard_normal(s) + 1j * g.standard_normal(s)) / np.sqrt(2)).astype(np.complex64)
    p = DevicePlan("c2c", prec, s)
    X = p.c2c(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel_l2(X.ravel(), O.fftn(x.astype(np.complex128), s)) <= F32_TOL
    back = p.c2c(torch.from_numpy(X).cuda(), inverse=True).cpu().numpy()
    assert rel_l2(back, x) <= 2 * F32_TOL


def test_psd_and_spectrogram_f64(golden):
    from fft_b200 import gofft as G
    for n in [7, 8, 15, 32, 1024]:
        x = rng(n).standard_normal(n)
        assert rel_l2(G.PSD(x, 0.1), O.psd(x, 0.1)) <= F64_TOL
    for seg, ov in [(8, 4), (32, 20), (2048, 1536), (15, 3)]:
        x = rng(seg).standard_normal(20000)
        w = O.hann(seg)
        frames = G.Spectrogram(x, seg, ov, w, 0.5)
        want = O.spectrogram(x, seg, ov, w, 0.5)
        assert len(frames) == want.shape[0]
        assert rel_l2(np.array(frames), want) <= F64_TOL
    got = G.Spectrogram(golden["spec_in"], 32, 20, golden["spec_win"], 1.0)
    np.testing.assert_allclose(np.array(got), golden["spec_out"], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("prec", ["f32", "f32mixed"])
def test_device_spectrogram_fp32(prec):
    from fft_b200.device import spectrogram
    x = rng(3).standard_normal(1 << 16).astype(np.float32)
    w = O.hann(2048).astype(np.float32)
    got = spectrogram(torch.from_numpy(x).cuda(), 2048, 1536, torch.from_numpy(w).cuda(), 1.0, prec)
    want = O.spectrogram(x.astype(np.float64), 2048, 1536, w.astype(np.float64), 1.0)
    assert got.shape == want.shape
    assert rel_l2(got.cpu().numpy(), want) <= F32_TOL


@pytest.mark.parametrize("prec", ["f64", "f32mixed"])
@pytest.mark.parametrize("shape,batch,gap", [([40, 64, 96], 1, 0), ([64, 96], 40, 0), ([20, 32, 48], 2, 5),
                                            ([6, 5, 64, 1009], 1, 0), ([10, 360, 48], 3, 0)])
def test_fftn_plane_blocks(prec, shape, batch, gap, small_l2_blocks):
    """Complex N-D transforms whose last two axes run per L2 block of planes
    on two lanes (a small block budget forces several blocks), against the
    oracle: merged and gapped batches, prime and smooth axes."""
    from fft_b200.device import DevicePlan
    n = int(np.prod(shape))
    dist = n + gap
    g = rng(n + batch)
    flat = g.standard_normal(batch * dist) + 1j * g.standard_normal(batch * dist)
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    tol = F64_TOL if prec == "f64" else F32_TOL
    p = DevicePlan("c2c", prec, shape, batch=batch, idist=dist, odist=dist)
    x = torch.from_numpy(flat).to(cdt).cuda()
    for inverse in (False, True):
        y = torch.zeros_like(x)
        p.c2c(x, out=y, inverse=inverse)
        got = y.cpu().numpy()
        for b in range(batch):
            want = O.fftn(flat[b * dist:b * dist + n], shape, inverse=inverse)
            assert rel_l2(got[b * dist:b * dist + n], want) <= tol, (shape, b, inverse)
