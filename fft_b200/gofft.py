"""The go-fft/fft API over the B200 engine, call for call.

Each name here is the reference's exported identifier with the same argument
meaning, normalisation and error behaviour; host arrays are numpy complex128
or float64 (the Go types complex128 and float64).  Where the reference panics
(bad shapes, bad spectrogram arguments) this raises :class:`GoPanic` with the
reference's panic text.  All arithmetic runs in libgofft_b200.so on the GPU.

Reference: plan.go, realplan.go, fft.go, rfft.go, rfft2.go, ndfft.go,
freq.go, window.go.
"""
import ctypes

import numpy as np

from ._lib import GOFFT_EINVAL, GOFFT_OK, GoFFTError, last_error, lib


class GoPanic(Exception):
    """Raised where the Go API panics (the message is the panic text)."""


def _call(status):
    if status == GOFFT_OK:
        return
    msg = last_error()
    if status == GOFFT_EINVAL and msg.startswith("fft:"):
        raise GoPanic(msg)
    raise GoFFTError(status, msg)


def _c128(x):
    return np.ascontiguousarray(x, dtype=np.complex128)


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a.size else None


class Plan:
    """A reusable transform of a fixed length (plan.go:19-30).  One plan
    serves FFT and IFFT and is safe for concurrent use."""

    def __init__(self, handle, n, owned=True):
        self._h = handle
        self._n = n
        self._owned = owned

    def Len(self):
        """plan.go:86"""
        return int(lib().gofft_plan_len(self._h)) if self._h else self._n

    def FFT(self, dst, src):
        """plan.go:91-94: forward DFT of src into dst (dst may alias src)."""
        self._check(dst, src)
        _call(lib().gofft_plan_fft(self._h, _ptr(dst), _ptr(src)))
        return dst

    def IFFT(self, dst, src):
        """plan.go:98-109: inverse DFT normalised by 1/N."""
        self._check(dst, src)
        _call(lib().gofft_plan_ifft(self._h, _ptr(dst), _ptr(src)))
        return dst

    def _check(self, dst, src):
        for a in (dst, src):
            if not (isinstance(a, np.ndarray) and a.dtype == np.complex128 and a.flags.c_contiguous):
                raise TypeError("dst and src must be contiguous complex128 arrays")
            if a.size != self._n:
                raise ValueError("dst and src must have length Len()")

    def __del__(self):
        try:
            if self._owned and self._h:
                lib().gofft_plan_destroy(self._h)
        except Exception:
            pass


def NewPlan(n):
    """plan.go:42-73"""
    h = ctypes.c_void_p()
    _call(lib().gofft_new_plan(int(n), ctypes.byref(h)))
    return Plan(h, int(n))


def cachedPlan(n):
    """plan.go:301-317: the memoised plan for n (same handle every call)."""
    h = ctypes.c_void_p()
    _call(lib().gofft_cached_plan(int(n), ctypes.byref(h)))
    return Plan(h, int(n), owned=False)


class RealPlan:
    """A reusable real-input transform (realplan.go:17-33)."""

    def __init__(self, handle, n):
        self._h = handle
        self._n = n

    def Len(self):
        return self._n

    def RFFT(self, dst, src):
        """realplan.go:77-116: n/2+1 bins of the real signal src."""
        src = np.asarray(src)
        if src.dtype != np.float64 or src.size != self._n or not src.flags.c_contiguous:
            raise ValueError("src must be contiguous float64 of length Len()")
        if dst.dtype != np.complex128 or dst.size < self._n // 2 + 1:
            raise ValueError("dst must be complex128 of length Len()/2+1")
        _call(lib().gofft_real_plan_rfft(self._h, _ptr(dst), _ptr(src)))
        return dst[: self._n // 2 + 1] if self._n else dst[:0]

    def IRFFT(self, dst, src):
        """realplan.go:181-192: reads min(len(src), n/2+1) bins."""
        src = _c128(src)
        if dst.dtype != np.float64 or dst.size != self._n or not dst.flags.c_contiguous:
            raise ValueError("dst must be contiguous float64 of length Len()")
        _call(lib().gofft_real_plan_irfft(self._h, _ptr(dst), _ptr(src), src.size))
        return dst

    def __del__(self):
        try:
            if self._h:
                lib().gofft_plan_destroy(self._h)
        except Exception:
            pass


def NewRealPlan(n):
    """realplan.go:37-58"""
    h = ctypes.c_void_p()
    _call(lib().gofft_new_real_plan(int(n), ctypes.byref(h)))
    return RealPlan(h, int(n))


def FFT(x):
    """fft.go:14-23"""
    x = _c128(x)
    out = np.zeros(x.size, dtype=np.complex128)
    _call(lib().gofft_fft(_ptr(x), x.size, _ptr(out)))
    return out


def IFFT(x):
    """fft.go:31-40"""
    x = _c128(x)
    out = np.zeros(x.size, dtype=np.complex128)
    _call(lib().gofft_ifft(_ptr(x), x.size, _ptr(out)))
    return out


def FFTReal(x):
    """fft.go:45-51"""
    x = _f64(x)
    out = np.zeros(x.size, dtype=np.complex128)
    _call(lib().gofft_fft_real(_ptr(x), x.size, _ptr(out)))
    return out


def RFFT(x):
    """rfft.go:19-26"""
    x = _f64(x)
    out = np.zeros(x.size // 2 + 1 if x.size else 0, dtype=np.complex128)
    _call(lib().gofft_rfft(_ptr(x), x.size, _ptr(out)))
    return out


def IRFFT(spectrum, n):
    """rfft.go:39-45"""
    s = _c128(spectrum)
    if n <= 0:
        return np.zeros(0)
    out = np.zeros(n, dtype=np.float64)
    _call(lib().gofft_irfft(_ptr(s), s.size, int(n), _ptr(out)))
    return out


def _shape(shape):
    sh = (ctypes.c_int64 * max(1, len(shape)))(*[int(s) for s in shape])
    return sh


def FFTN(data, shape):
    """ndfft.go:22-24"""
    d = _c128(data).reshape(-1)
    out = np.zeros(d.size, dtype=np.complex128)
    _call(lib().gofft_fftn(_ptr(d), d.size, _shape(shape), len(shape), _ptr(out)))
    return out


def IFFTN(data, shape):
    """ndfft.go:31-33"""
    d = _c128(data).reshape(-1)
    out = np.zeros(d.size, dtype=np.complex128)
    _call(lib().gofft_ifftn(_ptr(d), d.size, _shape(shape), len(shape), _ptr(out)))
    return out


def FFT2(data, shape):
    """ndfft.go:37-39"""
    d = _c128(data).reshape(-1)
    out = np.zeros(d.size, dtype=np.complex128)
    _call(lib().gofft_fft2(_ptr(d), d.size, int(shape[0]), int(shape[1]), _ptr(out)))
    return out


def IFFT2(data, shape):
    """ndfft.go:43-45"""
    d = _c128(data).reshape(-1)
    out = np.zeros(d.size, dtype=np.complex128)
    _call(lib().gofft_ifft2(_ptr(d), d.size, int(shape[0]), int(shape[1]), _ptr(out)))
    return out


def RFFT2(data, shape):
    """rfft2.go:22-74"""
    d = _f64(data).reshape(-1)
    rows, cols = int(shape[0]), int(shape[1])
    n = rows * (cols // 2 + 1) if rows > 0 and cols > 0 else 0
    out = np.zeros(max(n, 0), dtype=np.complex128)
    _call(lib().gofft_rfft2(_ptr(d), d.size, rows, cols, _ptr(out)))
    return out


def IRFFT2(data, shape):
    """rfft2.go:87-138"""
    d = _c128(data).reshape(-1)
    rows, cols = int(shape[0]), int(shape[1])
    out = np.zeros(max(rows * cols, 0) if rows > 0 and cols > 0 else 0, dtype=np.float64)
    _call(lib().gofft_irfft2(_ptr(d), d.size, rows, cols, _ptr(out)))
    return out


def Hann(n):
    """window.go:20-22"""
    if n <= 0:
        return np.zeros(0)
    out = np.zeros(n)
    _call(lib().gofft_hann(int(n), _ptr(out)))
    return out


def _window(fn, n):
    if n <= 0:
        return np.zeros(0)
    out = np.zeros(n)
    _call(fn(int(n), _ptr(out)))
    return out


def Hamming(n):
    """window.go:29-31"""
    return _window(lib().gofft_hamming, n)


def Blackman(n):
    """window.go:38-40"""
    return _window(lib().gofft_blackman, n)


def BlackmanHarris(n):
    """window.go:48-50"""
    return _window(lib().gofft_blackman_harris, n)


def Bartlett(n):
    """window.go:86-100"""
    return _window(lib().gofft_bartlett, n)


def FFTFreq(n, d):
    """freq.go:17-37"""
    if n <= 0:
        return np.zeros(0)
    out = np.zeros(n)
    _call(lib().gofft_fftfreq(int(n), float(d), _ptr(out)))
    return out


def RFFTFreq(n, d):
    """freq.go:46-56"""
    if n <= 0:
        return np.zeros(0)
    out = np.zeros(n // 2 + 1)
    _call(lib().gofft_rfftfreq(int(n), float(d), _ptr(out)))
    return out


def PSD(x, d):
    """freq.go:69-90"""
    x = _f64(x)
    if x.size == 0:
        return np.zeros(0)
    out = np.zeros(x.size // 2 + 1)
    _call(lib().gofft_psd(_ptr(x), x.size, float(d), _ptr(out)))
    return out


def Spectrogram(x, segment, overlap, window, d):
    """freq.go:107-127: returns a list of frames (None when no full frame
    fits, as the reference returns a nil slice)."""
    x = _f64(x)
    w = _f64(window)
    nf = ctypes.c_int64()
    _call(lib().gofft_spectrogram(_ptr(x), x.size, int(segment), int(overlap), _ptr(w), w.size, float(d),
                                  None, ctypes.byref(nf)))
    if nf.value == 0:
        return None
    out = np.zeros((nf.value, int(segment) // 2 + 1))
    _call(lib().gofft_spectrogram(_ptr(x), x.size, int(segment), int(overlap), _ptr(w), w.size, float(d),
                                  _ptr(out), ctypes.byref(nf)))
    return [row for row in out]
