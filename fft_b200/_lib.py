"""Loads libgofft_b200.so (built in-tree by ``fft_b200.build``) and declares
the C-ABI of ``include/gofft.h``.

There is no fallback: if the library is missing or fails to load, every
entry point raises.  The library is the product; nothing here computes a
transform in Python.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgofft_b200.so")

GOFFT_OK, GOFFT_EINVAL, GOFFT_ENOMEM, GOFFT_ECUDA, GOFFT_ETIMEOUT, GOFFT_EUNSUPPORTED = range(6)
GOFFT_C2C, GOFFT_R2C = 0, 1
GOFFT_F64, GOFFT_F32, GOFFT_F32MIXED = 0, 1, 2

_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.c_int64
_i64p = ctypes.POINTER(ctypes.c_int64)
_pp = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); mirrors include/gofft.h
SIGNATURES = {
    "gofft_last_error": (ctypes.c_char_p, []),
    "gofft_version": (ctypes.c_char_p, []),
    "gofft_new_plan": (ctypes.c_int, [_i64, _pp]),
    "gofft_cached_plan": (ctypes.c_int, [_i64, _pp]),
    "gofft_plan_len": (_i64, [_vp]),
    "gofft_plan_fft": (ctypes.c_int, [_vp, _vp, _vp]),
    "gofft_plan_ifft": (ctypes.c_int, [_vp, _vp, _vp]),
    "gofft_new_real_plan": (ctypes.c_int, [_i64, _pp]),
    "gofft_real_plan_rfft": (ctypes.c_int, [_vp, _vp, _vp]),
    "gofft_real_plan_irfft": (ctypes.c_int, [_vp, _vp, _vp, _i64]),
    "gofft_fft": (ctypes.c_int, [_vp, _i64, _vp]),
    "gofft_ifft": (ctypes.c_int, [_vp, _i64, _vp]),
    "gofft_fft_real": (ctypes.c_int, [_vp, _i64, _vp]),
    "gofft_rfft": (ctypes.c_int, [_vp, _i64, _vp]),
    "gofft_irfft": (ctypes.c_int, [_vp, _i64, _i64, _vp]),
    "gofft_fftn": (ctypes.c_int, [_vp, _i64, _i64p, ctypes.c_int, _vp]),
    "gofft_ifftn": (ctypes.c_int, [_vp, _i64, _i64p, ctypes.c_int, _vp]),
    "gofft_fft2": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp]),
    "gofft_ifft2": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp]),
    "gofft_rfft2": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp]),
    "gofft_irfft2": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp]),
    "gofft_hann": (ctypes.c_int, [_i64, _vp]),
    "gofft_psd": (ctypes.c_int, [_vp, _i64, ctypes.c_double, _vp]),
    "gofft_spectrogram": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _i64, ctypes.c_double, _vp, _i64p]),
    "gofft_plan_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _i64p, ctypes.c_int, _i64, _i64, _i64,
                                         _i64, _i64, _pp]),
    "gofft_plan_destroy": (ctypes.c_int, [_vp]),
    "gofft_plan_workspace_size": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_size_t)]),
    "gofft_plan_describe": (_i64, [_vp, ctypes.c_char_p, _i64]),
    "gofft_exec_c2c": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "gofft_exec_r2c": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "gofft_exec_c2r": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp]),
    "gofft_exec_c2c_noalloc": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "gofft_vjp_c2c": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "gofft_vjp_r2c": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "gofft_vjp_c2r": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "gofft_filter2_forward": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "gofft_vjp_filter2": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gofft_exec_c2c_host": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    "gofft_exec_r2c_host": (ctypes.c_int, [_vp, _vp, _vp]),
    "gofft_exec_c2r_host": (ctypes.c_int, [_vp, _vp, _i64, _vp]),
    "gofft_plan_table": (_i64, [_vp, ctypes.c_int, _i64p, _i64]),
    "gofft_spectrogram_device": (ctypes.c_int, [ctypes.c_int, _vp, _i64, _i64, _i64, _vp, ctypes.c_double, _vp,
                                                _i64p, _vp]),
    "gofft_uneven_create": (ctypes.c_int, [ctypes.c_int, _i64p, _i64, _i64p, _i64p, _pp]),
    "gofft_uneven_destroy": (ctypes.c_int, [_vp]),
    "gofft_uneven_exec": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "gofft_uneven_status": (ctypes.c_int, [_vp]),
    "gofft_uneven_set": (ctypes.c_int, [_vp, ctypes.c_int, _i64]),
    "gofft_uneven_describe": (_i64, [_vp, ctypes.c_char_p, _i64]),
    "gofft_graph_begin": (ctypes.c_int, [_vp]),
    "gofft_graph_end": (ctypes.c_int, [_vp, _pp]),
    "gofft_graph_launch": (ctypes.c_int, [_vp, _vp]),
    "gofft_graph_destroy": (ctypes.c_int, [_vp]),
    "gofft_launch_count": (_i64, []),
    "gofft_timing_enable": (ctypes.c_int, [ctypes.c_int]),
    "gofft_timing_report": (_i64, [ctypes.c_char_p, _i64]),
    "gofft_set_lines_per_cta": (ctypes.c_int, [ctypes.c_int, _i64, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gofft_set_pipelined": (ctypes.c_int, [ctypes.c_int, _i64, ctypes.c_int, ctypes.c_int]),
    "gofft_set_l2_block_bytes": (ctypes.c_int, [_i64]),
    "gofft_set_lanes": (ctypes.c_int, [ctypes.c_int]),
    "gofft_set_tma_pipeline": (ctypes.c_int, [ctypes.c_int]),
    "gofft_set_dependent_launch": (ctypes.c_int, [ctypes.c_int]),
    "gofft_pipeline_status": (ctypes.c_int, []),
    "gofft_set_schedule": (ctypes.c_int, [ctypes.c_int, _i64, ctypes.c_int]),
    "gofft_hamming": (ctypes.c_int, [_i64, _vp]),
    "gofft_blackman": (ctypes.c_int, [_i64, _vp]),
    "gofft_blackman_harris": (ctypes.c_int, [_i64, _vp]),
    "gofft_bartlett": (ctypes.c_int, [_i64, _vp]),
    "gofft_fftfreq": (ctypes.c_int, [_i64, ctypes.c_double, _vp]),
    "gofft_rfftfreq": (ctypes.c_int, [_i64, ctypes.c_double, _vp]),
    "gofft_window_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _i64, _vp, _vp]),
    "gofft_spectrogram_window_device": (ctypes.c_int, [ctypes.c_int, _vp, _i64, _i64, _i64, ctypes.c_int,
                                                       ctypes.c_double, _vp, _i64p, _vp]),
    "gofft_get_schedule": (ctypes.c_int, [ctypes.c_int, _i64]),
    "gofft_autotune": (_i64, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _i64, ctypes.c_char_p, _i64]),
    "gofft_autotune_uneven": (_i64, [ctypes.c_int, _vp, _i64, ctypes.c_char_p, _i64]),
    "gofft_wisdom_export": (_i64, [ctypes.c_char_p, _i64]),
    "gofft_wisdom_import": (ctypes.c_int, [ctypes.c_char_p]),
    "gofft_wisdom_forget": (ctypes.c_int, []),
}

_lib = None


class GoFFTError(RuntimeError):
    """A non-OK status from the C-ABI."""

    def __init__(self, status, msg):
        super().__init__("gofft status %d: %s" % (status, msg))
        self.status = status
        self.msg = msg


def lib():
    """The loaded library; raises if it is absent (build it with
    ``python -m fft_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libgofft_b200.so is not built (run python -m fft_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    return lib().gofft_last_error().decode()


def check(status):
    if status != GOFFT_OK:
        raise GoFFTError(status, last_error())
    return status


def launch_count():
    """Engine kernels launched by this process so far."""
    return int(lib().gofft_launch_count())


def timing_enable(on=True):
    lib().gofft_timing_enable(1 if on else 0)


def timing_report():
    """Per-kernel CUDA-event timings since the last call (list of dicts)."""
    import json
    n = lib().gofft_timing_report(None, 0)
    buf = ctypes.create_string_buffer(int(n) + 1)
    lib().gofft_timing_report(buf, n + 1)
    return json.loads(buf.value.decode() or "[]")
