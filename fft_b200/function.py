"""Differentiable transforms: the Forward/Backward ``Function`` interface and
its torch.autograd bridge.  No counterpart in go-fft/fft (the library has no
differentiation); the adjoints are the library's own kernels
(gofft_vjp_* in include/gofft.h), never torch's.

    f = SpectralFilter2("f32mixed", 512, 512, batch=32)
    y = f.Forward(x, H)          # IRFFT2(H * RFFT2(x)) per image
    dx, dH = f.Backward(2 * y)   # gradients of sum(y**2)

    y = apply(f, x, H)           # the same through torch.autograd
    (y ** 2).sum().backward()    # x.grad, H.grad from f.Backward

A Function object keeps what its last Forward saved for the next Backward
(like torch's ctx): one Forward per Backward, one call in flight at a time.
Complex gradients follow torch's convention for a real loss: dL/dRe + i dL/dIm.
"""
import torch

from .device import DevicePlan


class Function:
    """Forward computes outputs and saves what Backward needs; Backward maps
    the gradients of the outputs to the gradients of the inputs (one per
    input, None where an input takes no gradient)."""

    def Forward(self, *inputs):
        raise NotImplementedError

    def Backward(self, *grads):
        raise NotImplementedError


class FFT(Function):
    """Batched complex transform of a row-major shape (rank >= 1); inverse
    selects the normalised inverse.  Backward: FFT^H = N IFFT, IFFT^H = FFT/N."""

    def __init__(self, precision, shape, batch=1, inverse=False):
        self.plan = DevicePlan("c2c", precision, shape, batch)
        self.inverse = bool(inverse)

    def Forward(self, x):
        return self.plan.c2c(x.contiguous(), inverse=self.inverse)

    def Backward(self, g):
        return self.plan.vjp_c2c(g.contiguous(), inverse=self.inverse)


class IFFT(FFT):
    def __init__(self, precision, shape, batch=1):
        super().__init__(precision, shape, batch, inverse=True)


class RFFT(Function):
    """Batched real forward transform (rank 1, or rank 2 = RFFT2).  Backward
    is N IRFFT(g / w) with the edge-bin weights w of the last axis."""

    def __init__(self, precision, shape, batch=1):
        self.plan = DevicePlan("r2c", precision, shape, batch)

    def Forward(self, x):
        return self.plan.r2c(x.contiguous())

    def Backward(self, g):
        return self.plan.vjp_r2c(g.contiguous())


class IRFFT(Function):
    """Batched real inverse transform (all n/2+1 bins read; rank 1, or rank
    2 = IRFFT2).  Backward is (w / N) RFFT(g)."""

    def __init__(self, precision, shape, batch=1):
        self.plan = DevicePlan("r2c", precision, shape, batch)

    def Forward(self, X):
        return self.plan.c2r(X.contiguous())

    def Backward(self, g):
        return self.plan.vjp_c2r(g.contiguous())


def RFFT2(precision, rows, cols, batch=1):
    return RFFT(precision, [rows, cols], batch)


def IRFFT2(precision, rows, cols, batch=1):
    return IRFFT(precision, [rows, cols], batch)


class SpectralFilter2(Function):
    """y_b = IRFFT2(H * RFFT2(x_b)) for a batch of R x C real images and one
    R x (C/2+1) complex filter H, fused into three passes per block of
    images.  Backward(g) = (dx, dH):
        dx = IRFFT2(conj(H) * RFFT2(g)),
        dH = sum_b conj(RFFT2(x_b)) * (w / (R C)) * RFFT2(g_b)."""

    def __init__(self, precision, rows, cols, batch=1):
        self.plan = DevicePlan("r2c", precision, [rows, cols], batch)
        self.saved = None
        self.H = None
        self.need_dh = True

    def Forward(self, x, H, need_dh=True):
        x = x.contiguous()
        H = H.contiguous()
        self.need_dh = bool(need_dh)
        self.saved = None
        if self.need_dh:
            self.saved = torch.empty((self.plan.batch, self.plan.bins), dtype=self.plan.cdtype, device=x.device)
        self.H = H
        return self.plan.filter2(x, H, saved=self.saved)

    def Backward(self, g, need_dx=True):
        g = g.contiguous()
        # the saved spectra double as the dH scratch: one Backward per Forward
        dx, dH = self.plan.vjp_filter2(g, self.H, saved=self.saved, scratch=self.saved, dx=need_dx,
                                       dH=self.need_dh)
        self.saved = None
        return dx, dH


class _Bridge(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fn, *inputs):
        ctx.fn = fn
        ctx.n_in = len(inputs)
        if isinstance(fn, SpectralFilter2):
            return fn.Forward(inputs[0], inputs[1], need_dh=ctx.needs_input_grad[2])
        return fn.Forward(*inputs)

    @staticmethod
    def backward(ctx, *grads):
        fn = ctx.fn
        if isinstance(fn, SpectralFilter2):
            dx, dH = fn.Backward(grads[0], need_dx=ctx.needs_input_grad[1])
            return None, dx, dH
        out = fn.Backward(*grads)
        if not isinstance(out, tuple):
            out = (out,)
        return (None,) + out


def apply(fn, *inputs):
    """Runs fn.Forward under torch.autograd; backward() calls fn.Backward."""
    return _Bridge.apply(fn, *inputs)
