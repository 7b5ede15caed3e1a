"""ctypes wrapper over the C restatement of go-fft/fft (``gofft_oracle.c``).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this module; it is the checker, never
the thing measured as the product.  Arrays are numpy complex128 / float64.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libgofft_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_i64p = ctypes.POINTER(ctypes.c_int64)

OR_TRIVIAL, OR_IT, OR_CT, OR_RADER, OR_BLUESTEIN = range(5)
ENGINE_NAMES = {0: "trivial", 1: "it", 2: "ct", 3: "rader", 4: "bluestein"}


def build():
    """Compile the oracle with its Makefile (gcc -O2 -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        sig = {
            "or_engine": (ctypes.c_int, [ctypes.c_int]),
            "or_factors_small": (ctypes.c_int, [ctypes.c_int]),
            "or_factorize": (ctypes.c_int, [ctypes.c_int, _ip]),
            "or_next_smooth_conv": (ctypes.c_int, [ctypes.c_int]),
            "or_conv_cost": (ctypes.c_int, [ctypes.c_int, _dp]),
            "or_best_conv_len": (ctypes.c_int, [ctypes.c_int]),
            "or_is_prime": (ctypes.c_int, [ctypes.c_int]),
            "or_primitive_root": (ctypes.c_int, [ctypes.c_int]),
            "or_it_radices": (ctypes.c_int, [ctypes.c_int, _ip]),
            "or_rev_pos": (None, [ctypes.c_int, _ip]),
            "or_bit_reverse_perm": (None, [ctypes.c_int, _ip]),
            "or_rader_info": (ctypes.c_int, [ctypes.c_int, _ip, _ip, _ip, _ip]),
            "or_bluestein_m": (ctypes.c_int, [ctypes.c_int]),
            "or_chirp_index": (None, [ctypes.c_int, _i64p]),
            "or_fft": (None, [ctypes.c_int, _dp, _dp]),
            "or_ifft": (None, [ctypes.c_int, _dp, _dp]),
            "or_execute": (None, [ctypes.c_int, _dp, _dp, ctypes.c_int]),
            "or_bluestein_transform": (None, [ctypes.c_int, _dp, _dp, ctypes.c_int]),
            "or_rader_transform": (None, [ctypes.c_int, _dp, _dp, ctypes.c_int]),
            "or_rfft": (None, [ctypes.c_int, _dp, _dp]),
            "or_irfft": (None, [ctypes.c_int, _dp, _dp, ctypes.c_int]),
            "or_set_workers": (None, [ctypes.c_int]),
            "or_get_workers": (ctypes.c_int, []),
            "or_fftn": (None, [_dp, _dp, _ip, ctypes.c_int, ctypes.c_int]),
            "or_rfft2": (None, [_dp, _dp, ctypes.c_int, ctypes.c_int]),
            "or_irfft2": (None, [_dp, _dp, ctypes.c_int64, ctypes.c_int, ctypes.c_int]),
            "or_cosine_window": (None, [ctypes.c_int, _dp, ctypes.c_int, _dp]),
            "or_hann": (None, [ctypes.c_int, _dp]),
            "or_psd": (None, [ctypes.c_int, _dp, ctypes.c_double, _dp]),
            "or_spectrogram": (ctypes.c_int, [_dp, ctypes.c_int64, ctypes.c_int, ctypes.c_int, _dp,
                                              ctypes.c_double, _dp]),
            "or_batch_fft": (None, [ctypes.c_int, ctypes.c_int64, _dp, _dp, ctypes.c_int]),
            "or_batch_rfft2_roundtrip": (None, [ctypes.c_int64, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                                _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _c128(x):
    return np.ascontiguousarray(x, dtype=np.complex128)


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64)


# ---- integer helpers --------------------------------------------------------

def engine(n):
    return lib().or_engine(n)


def factors_small(n):
    return bool(lib().or_factors_small(n))


def factorize(n):
    buf = (ctypes.c_int * 64)()
    c = lib().or_factorize(n, buf)
    return list(buf[:c])


def next_smooth_conv(lo):
    return lib().or_next_smooth_conv(lo)


def conv_cost(m):
    c = ctypes.c_double()
    ok = lib().or_conv_cost(m, ctypes.byref(c))
    return c.value, bool(ok)


def best_conv_len(lo):
    return lib().or_best_conv_len(lo)


def is_prime(n):
    return bool(lib().or_is_prime(n))


def primitive_root(p):
    return lib().or_primitive_root(p)


def it_radices(n):
    buf = (ctypes.c_int * 64)()
    c = lib().or_it_radices(n, buf)
    return list(buf[:c])


def rev_pos(n):
    out = np.zeros(n, dtype=np.int32)
    lib().or_rev_pos(n, out.ctypes.data_as(_ip))
    return out


def bit_reverse_perm(n):
    out = np.zeros(n, dtype=np.int32)
    lib().or_bit_reverse_perm(n, out.ctypes.data_as(_ip))
    return out


def rader_info(n):
    q = n - 1
    perm = np.zeros(q, dtype=np.int32)
    iperm = np.zeros(q, dtype=np.int32)
    cyc = ctypes.c_int()
    g = ctypes.c_int()
    cl = lib().or_rader_info(n, ctypes.byref(cyc), ctypes.byref(g), perm.ctypes.data_as(_ip),
                             iperm.ctypes.data_as(_ip))
    return {"cl": cl, "cyclic": bool(cyc.value), "g": g.value, "perm": perm, "iperm": iperm}


def bluestein_m(n):
    return lib().or_bluestein_m(n)


def chirp_index(n):
    out = np.zeros(n, dtype=np.int64)
    lib().or_chirp_index(n, out.ctypes.data_as(_i64p))
    return out


# ---- transforms -------------------------------------------------------------

def fft(x):
    x = _c128(x)
    out = np.empty_like(x)
    if x.size:
        lib().or_fft(x.size, _d(out.view(np.float64)), _d(x.view(np.float64)))
    return out


def ifft(x):
    x = _c128(x)
    out = np.empty_like(x)
    if x.size:
        lib().or_ifft(x.size, _d(out.view(np.float64)), _d(x.view(np.float64)))
    return out


def execute(x, inverse=False):
    x = _c128(x)
    out = np.empty_like(x)
    lib().or_execute(x.size, _d(out.view(np.float64)), _d(x.view(np.float64)), int(inverse))
    return out


def bluestein(x, inverse=False):
    x = _c128(x)
    out = np.empty_like(x)
    lib().or_bluestein_transform(x.size, _d(out.view(np.float64)), _d(x.view(np.float64)),
                                 int(inverse))
    return out


def rader(x, inverse=False):
    x = _c128(x)
    out = np.empty_like(x)
    lib().or_rader_transform(x.size, _d(out.view(np.float64)), _d(x.view(np.float64)), int(inverse))
    return out


def rfft(x):
    x = _f64(x)
    n = x.size
    out = np.zeros(n // 2 + 1 if n else 0, dtype=np.complex128)
    if n:
        lib().or_rfft(n, _d(out.view(np.float64)), _d(x))
    return out


def irfft(spec, n):
    spec = _c128(spec)
    if n <= 0:
        return np.zeros(0)
    out = np.zeros(n, dtype=np.float64)
    lib().or_irfft(n, _d(out), _d(spec.view(np.float64)) if spec.size else None, spec.size)
    return out


def set_workers(w):
    lib().or_set_workers(int(w))


def get_workers():
    return lib().or_get_workers()


def fftn(x, shape, inverse=False):
    x = _c128(x).reshape(-1)
    sh = (ctypes.c_int * max(1, len(shape)))(*shape)
    out = np.empty_like(x)
    lib().or_fftn(_d(out.view(np.float64)), _d(x.view(np.float64)), sh, len(shape), int(inverse))
    return out


def ifftn(x, shape):
    return fftn(x, shape, inverse=True)


def rfft2(x, rows, cols):
    x = _f64(x).reshape(-1)
    out = np.zeros(rows * (cols // 2 + 1), dtype=np.complex128)
    lib().or_rfft2(_d(out.view(np.float64)), _d(x), rows, cols)
    return out


def irfft2(spec, rows, cols):
    spec = _c128(spec).reshape(-1)
    out = np.zeros(rows * cols, dtype=np.float64)
    ptr = _d(spec.view(np.float64)) if spec.size else None
    lib().or_irfft2(_d(out), ptr, spec.size, rows, cols)
    return out


def cosine_window(n, coeffs):
    if n <= 0:
        return np.zeros(0)
    a = _f64(coeffs)
    out = np.zeros(n)
    lib().or_cosine_window(n, _d(a), a.size, _d(out))
    return out


def hann(n):
    if n <= 0:
        return np.zeros(0)
    out = np.zeros(n)
    lib().or_hann(n, _d(out))
    return out


def psd(x, d):
    x = _f64(x)
    if x.size == 0:
        return np.zeros(0)
    out = np.zeros(x.size // 2 + 1)
    lib().or_psd(x.size, _d(x), float(d), _d(out))
    return out


def spectrogram(x, segment, overlap, window, d):
    x = _f64(x)
    w = _f64(window)
    frames = lib().or_spectrogram(_d(x), x.size, segment, overlap, _d(w), float(d), None)
    out = np.zeros((frames, segment // 2 + 1))
    if frames:
        lib().or_spectrogram(_d(x), x.size, segment, overlap, _d(w), float(d), _d(out))
    return out


def batch_fft(x, inverse=False):
    """``batch`` independent Plan.FFT/IFFT calls over the rows of x (2-D array)."""
    x = _c128(x)
    b, n = x.shape
    out = np.empty_like(x)
    lib().or_batch_fft(n, b, _d(out.view(np.float64)), _d(x.view(np.float64)), int(inverse))
    return out


def batch_rfft2_roundtrip(x):
    """RFFT2 then IRFFT2 of each image in x (batch, rows, cols)."""
    x = _f64(x)
    b, r, c = x.shape
    spec = np.zeros((b, r, c // 2 + 1), dtype=np.complex128)
    back = np.zeros_like(x)
    lib().or_batch_rfft2_roundtrip(b, r, c, _d(x), _d(spec.view(np.float64)), _d(back))
    return spec, back
