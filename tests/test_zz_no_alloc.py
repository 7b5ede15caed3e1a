"""The allocation-free complex transform (gofft_exec_c2c_noalloc), for callers
that cannot have device memory allocated while they run (graph capture,
memory owned by another allocator, no room for cudaMalloc's synchronisation).
It must agree with gofft_exec_c2c, call after call, using only the library's
built-in scratch array.  Collected last (file name) so that a failure here
does not hide the rest of the suite."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_l2, rng

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32mixed": 1e-6}


# multi-pass transforms that need scratch: the four-step split, and the four
# Rader passes of a convolution too long for a pair of CTAs (FP64 14411:
# cl = 29400 complex128, 470 KB)
@pytest.mark.parametrize("prec,n,batch", [("f32mixed", 65536, 4), ("f64", 16384, 8), ("f64", 14411, 3)])
def test_noalloc_matches_exec_c2c(prec, n, batch):
    from fft_b200._lib import check, lib
    from fft_b200.device import DevicePlan
    p = DevicePlan("c2c", prec, [n], batch=batch)
    assert p.workspace_bytes() > 0  # a transform that needs scratch
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    st = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        g = rng(100 + call)
        x = torch.from_numpy(g.standard_normal((batch, n)) + 1j * g.standard_normal((batch, n))).to(cdt).cuda()
        for inverse in (0, 1):
            ref = p.c2c(x, inverse=bool(inverse))
            got = torch.empty_like(x)
            check(lib().gofft_exec_c2c_noalloc(p.handle, ctypes.c_void_p(x.data_ptr()),
                                               ctypes.c_void_p(got.data_ptr()), inverse, ctypes.c_void_p(st)))
            torch.cuda.synchronize()
            err = rel_l2(got.cpu().numpy(), ref.cpu().numpy())
            assert err <= TOL[prec], (prec, n, call, inverse, err)


def test_noalloc_rejects_wrong_plans():
    from fft_b200._lib import GOFFT_EINVAL, GOFFT_EUNSUPPORTED, lib
    from fft_b200.device import DevicePlan
    x = torch.zeros(1, 64 * 64, dtype=torch.complex128, device="cuda")
    xp, st = ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    real = DevicePlan("r2c", "f64", [1024])
    assert lib().gofft_exec_c2c_noalloc(real.handle, xp, xp, 0, st) == GOFFT_EINVAL
    assert "complex-to-complex" in lib().gofft_last_error().decode()
    two_d = DevicePlan("c2c", "f64", [64, 64])
    assert lib().gofft_exec_c2c_noalloc(two_d.handle, xp, xp, 0, st) == GOFFT_EUNSUPPORTED


def test_noalloc_rejects_oversized():
    from fft_b200._lib import GOFFT_EINVAL, lib
    from fft_b200.device import DevicePlan
    p = DevicePlan("c2c", "f64", [65536], batch=64)  # needs more than the built-in scratch
    x = torch.zeros(64, 65536, dtype=torch.complex128, device="cuda")
    st = lib().gofft_exec_c2c_noalloc(p.handle, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), 0,
                                      None)
    assert st == GOFFT_EINVAL
    assert "scratch" in lib().gofft_last_error().decode()
