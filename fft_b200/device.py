"""Device-resident plans on torch tensors (plumbing only: torch owns the
memory and the stream; every transform runs in libgofft_b200.so).

    p = DevicePlan("c2c", "f64", [1024], batch=256)
    y = p.c2c(x)                    # x: complex128 cuda tensor (256, 1024)
    X = DevicePlan("r2c", "f32mixed", [512, 512], batch=32).r2c(img)
"""
import ctypes
import json

import torch

from ._lib import GOFFT_C2C, GOFFT_F32, GOFFT_F32MIXED, GOFFT_F64, GOFFT_R2C, check, lib

PRECISIONS = {"f64": GOFFT_F64, "f32": GOFFT_F32, "f32mixed": GOFFT_F32MIXED}
KINDS = {"c2c": GOFFT_C2C, "r2c": GOFFT_R2C}
CDT = {GOFFT_F64: torch.complex128, GOFFT_F32: torch.complex64, GOFFT_F32MIXED: torch.complex64}
RDT = {GOFFT_F64: torch.float64, GOFFT_F32: torch.float32, GOFFT_F32MIXED: torch.float32}


def _stream(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _need(t, dtype, what):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("%s must be a CUDA tensor" % what)
    if t.dtype != dtype:
        raise TypeError("%s must be %s, got %s" % (what, dtype, t.dtype))
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % what)


class DevicePlan:
    """A batched plan on the current CUDA device (gofft_plan_create)."""

    def __init__(self, kind, precision, shape, batch=1, istride=0, idist=0, ostride=0, odist=0):
        self.kind = KINDS[kind] if isinstance(kind, str) else int(kind)
        self.prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self.shape = [int(s) for s in shape]
        self.batch = int(batch)
        sh = (ctypes.c_int64 * len(self.shape))(*self.shape)
        h = ctypes.c_void_p()
        check(lib().gofft_plan_create(self.kind, self.prec, sh, len(self.shape), self.batch, istride, idist,
                                      ostride, odist, ctypes.byref(h)))
        self._h = h
        self.cdtype = CDT[self.prec]
        self.rdtype = RDT[self.prec]
        n = 1
        for s in self.shape:
            n *= s
        self.numel = n
        self.bins = n // self.shape[-1] * (self.shape[-1] // 2 + 1)

    @property
    def handle(self):
        return self._h

    def c2c(self, x, out=None, inverse=False, stream=None):
        _need(x, self.cdtype, "x")
        if out is None:
            out = torch.empty_like(x)
        _need(out, self.cdtype, "out")
        check(lib().gofft_exec_c2c(self._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                   1 if inverse else 0, _stream(stream)))
        return out

    def r2c(self, x, out=None, stream=None):
        _need(x, self.rdtype, "x")
        if out is None:
            out = torch.empty((self.batch, self.bins), dtype=self.cdtype, device=x.device)
        _need(out, self.cdtype, "out")
        check(lib().gofft_exec_r2c(self._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                   _stream(stream)))
        return out

    def c2r(self, X, out=None, nbins=0, stream=None):
        _need(X, self.cdtype, "X")
        if out is None:
            out = torch.empty((self.batch, self.numel), dtype=self.rdtype, device=X.device)
        _need(out, self.rdtype, "out")
        check(lib().gofft_exec_c2r(self._h, ctypes.c_void_p(X.data_ptr()), int(nbins),
                                   ctypes.c_void_p(out.data_ptr()), _stream(stream)))
        return out

    # adjoints (vector-Jacobian products): real inner product, so a complex
    # gradient holds dL/dRe + i dL/dIm
    def vjp_c2c(self, g, out=None, inverse=False, stream=None):
        _need(g, self.cdtype, "g")
        if out is None:
            out = torch.empty_like(g)
        _need(out, self.cdtype, "out")
        check(lib().gofft_vjp_c2c(self._h, ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                  1 if inverse else 0, _stream(stream)))
        return out

    def vjp_r2c(self, g, out=None, stream=None):
        """Adjoint of r2c: bins -> reals."""
        _need(g, self.cdtype, "g")
        if out is None:
            out = torch.empty((self.batch, self.numel), dtype=self.rdtype, device=g.device)
        _need(out, self.rdtype, "out")
        check(lib().gofft_vjp_r2c(self._h, ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                  _stream(stream)))
        return out

    def vjp_c2r(self, g, out=None, stream=None):
        """Adjoint of c2r (all bins read): reals -> bins."""
        _need(g, self.rdtype, "g")
        if out is None:
            out = torch.empty((self.batch, self.bins), dtype=self.cdtype, device=g.device)
        _need(out, self.cdtype, "out")
        check(lib().gofft_vjp_c2r(self._h, ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                  _stream(stream)))
        return out

    def filter2(self, x, H, out=None, saved=None, stream=None):
        """y = IRFFT2(H * RFFT2(x)) per image (rank-2 real plans); saved, if
        given, receives the spectra RFFT2(x) for the backward's dH."""
        _need(x, self.rdtype, "x")
        _need(H, self.cdtype, "H")
        if out is None:
            out = torch.empty_like(x)
        _need(out, self.rdtype, "out")
        sp = None
        if saved is not None:
            _need(saved, self.cdtype, "saved")
            sp = ctypes.c_void_p(saved.data_ptr())
        check(lib().gofft_filter2_forward(self._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(H.data_ptr()),
                                          ctypes.c_void_p(out.data_ptr()), sp, _stream(stream)))
        return out

    def vjp_filter2(self, g, H, saved=None, scratch=None, dx=True, dH=True, stream=None):
        """(dx, dH) of filter2 for the upstream gradient g; either may be
        skipped.  dH needs the forward's saved spectra; scratch defaults to a
        fresh buffer (pass saved itself to let it be overwritten)."""
        _need(g, self.rdtype, "g")
        _need(H, self.cdtype, "H")
        ox = torch.empty_like(g) if dx else None
        oh = torch.empty_like(H) if dH else None
        sp = sc = None
        if dH:
            if saved is None:
                raise ValueError("dH needs the saved spectra of the forward")
            _need(saved, self.cdtype, "saved")
            if scratch is None:
                scratch = torch.empty_like(saved)
            _need(scratch, self.cdtype, "scratch")
            sp, sc = ctypes.c_void_p(saved.data_ptr()), ctypes.c_void_p(scratch.data_ptr())
        check(lib().gofft_vjp_filter2(self._h, ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(H.data_ptr()), sp, sc,
                                      ctypes.c_void_p(ox.data_ptr()) if dx else None,
                                      ctypes.c_void_p(oh.data_ptr()) if dH else None, _stream(stream)))
        return ox, oh

    # host-pointer variants (copies inside the call): numpy or pinned tensors
    def c2c_host(self, x_ptr, out_ptr, inverse=False):
        check(lib().gofft_exec_c2c_host(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(out_ptr),
                                        1 if inverse else 0))

    def r2c_host(self, x_ptr, out_ptr):
        check(lib().gofft_exec_r2c_host(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(out_ptr)))

    def c2r_host(self, x_ptr, out_ptr, nbins=0):
        check(lib().gofft_exec_c2r_host(self._h, ctypes.c_void_p(x_ptr), int(nbins), ctypes.c_void_p(out_ptr)))

    def describe(self):
        n = lib().gofft_plan_describe(self._h, None, 0)
        buf = ctypes.create_string_buffer(int(n) + 1)
        lib().gofft_plan_describe(self._h, buf, n + 1)
        return json.loads(buf.value.decode())

    def table(self, which):
        n = lib().gofft_plan_table(self._h, int(which), None, 0)
        if n < 0:
            return None
        out = (ctypes.c_int64 * max(1, n))()
        lib().gofft_plan_table(self._h, int(which), out, n)
        return list(out[:n])

    def workspace_bytes(self):
        v = ctypes.c_size_t()
        check(lib().gofft_plan_workspace_size(self._h, ctypes.byref(v)))
        return v.value

    def close(self):
        if self._h:
            lib().gofft_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spectrogram(x, segment, overlap, window, d, precision="f64", stream=None):
    """Fused spectrogram (freq.go:107-127) of a device signal; returns a
    (frames, segment//2+1) tensor of one-sided densities."""
    prec = PRECISIONS[precision]
    _need(x, RDT[prec], "x")
    _need(window, RDT[prec], "window")
    nf = ctypes.c_int64()
    check(lib().gofft_spectrogram_device(prec, ctypes.c_void_p(x.data_ptr()), x.numel(), int(segment),
                                         int(overlap), ctypes.c_void_p(window.data_ptr()), float(d), None,
                                         ctypes.byref(nf), _stream(stream)))
    out = torch.empty((nf.value, int(segment) // 2 + 1), dtype=RDT[prec], device=x.device)
    if nf.value:
        check(lib().gofft_spectrogram_device(prec, ctypes.c_void_p(x.data_ptr()), x.numel(), int(segment),
                                             int(overlap), ctypes.c_void_p(window.data_ptr()), float(d),
                                             ctypes.c_void_p(out.data_ptr()), ctypes.byref(nf),
                                             _stream(stream)))
    return out


WINDOWS = {"hann": 0, "hamming": 1, "blackman": 2, "blackmanharris": 3, "bartlett": 4}


def window(kind, n, precision="f64", stream=None):
    """A symmetric window (window.go:20-100) generated on the device."""
    prec = PRECISIONS[precision]
    out = torch.empty(int(n), dtype=RDT[prec], device="cuda")
    if n > 0:
        check(lib().gofft_window_device(prec, WINDOWS[kind], int(n), ctypes.c_void_p(out.data_ptr()),
                                        _stream(stream)))
    return out


def spectrogram_window(x, segment, overlap, kind, d, precision="f64", stream=None):
    """Fused spectrogram with a device-generated window of `kind`."""
    prec = PRECISIONS[precision]
    _need(x, RDT[prec], "x")
    nf = ctypes.c_int64()
    check(lib().gofft_spectrogram_window_device(prec, ctypes.c_void_p(x.data_ptr()), x.numel(), int(segment),
                                                int(overlap), WINDOWS[kind], float(d), None, ctypes.byref(nf),
                                                _stream(stream)))
    out = torch.empty((nf.value, int(segment) // 2 + 1), dtype=RDT[prec], device=x.device)
    if nf.value:
        check(lib().gofft_spectrogram_window_device(prec, ctypes.c_void_p(x.data_ptr()), x.numel(), int(segment),
                                                    int(overlap), WINDOWS[kind], float(d),
                                                    ctypes.c_void_p(out.data_ptr()), ctypes.byref(nf),
                                                    _stream(stream)))
    return out


class UnevenBatch:
    """Complex transforms of different lengths in one persistent launch
    (gofft_uneven_*).  Signals are packed back to back in one tensor unless
    offsets are given."""

    def __init__(self, precision, lengths, in_offsets=None, out_offsets=None):
        self.prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self.lengths = [int(n) for n in lengths]
        n = len(self.lengths)
        L = (ctypes.c_int64 * n)(*self.lengths)
        io = (ctypes.c_int64 * n)(*in_offsets) if in_offsets is not None else None
        oo = (ctypes.c_int64 * n)(*out_offsets) if out_offsets is not None else None
        h = ctypes.c_void_p()
        check(lib().gofft_uneven_create(self.prec, L, n, io, oo, ctypes.byref(h)))
        self._h = h
        self.cdtype = CDT[self.prec]

    def __call__(self, x, out=None, inverse=False, stream=None):
        _need(x, self.cdtype, "x")
        if out is None:
            out = torch.empty_like(x)
        check(lib().gofft_uneven_exec(self._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                      1 if inverse else 0, _stream(stream)))
        return out

    def status(self):
        return lib().gofft_uneven_status(self._h)

    def set(self, what, value):
        check(lib().gofft_uneven_set(self._h, int(what), int(value)))

    def describe(self):
        n = lib().gofft_uneven_describe(self._h, None, 0)
        buf = ctypes.create_string_buffer(int(n) + 1)
        lib().gofft_uneven_describe(self._h, buf, n + 1)
        return json.loads(buf.value.decode())

    def close(self):
        if self._h:
            lib().gofft_uneven_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """A captured sequence of engine calls on a (non-default) stream."""

    def __init__(self, stream):
        self.stream = stream
        self._h = None

    def __enter__(self):
        check(lib().gofft_graph_begin(ctypes.c_void_p(self.stream.cuda_stream)))
        return self

    def __exit__(self, *exc):
        h = ctypes.c_void_p()
        st = lib().gofft_graph_end(ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h))
        if exc[0] is None:
            check(st)
        self._h = h

    def replay(self):
        check(lib().gofft_graph_launch(self._h, ctypes.c_void_p(self.stream.cuda_stream)))

    def __del__(self):
        try:
            if self._h:
                lib().gofft_graph_destroy(self._h)
        except Exception:
            pass
