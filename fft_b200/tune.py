"""The autotuner and its wisdom (gofft_autotune / gofft_wisdom_* in the
C-ABI).  No counterpart in go-fft/fft, whose plans are fixed by its router.

    w = autotune("r2c", "f64", [1024, 1024], batch=32)   # times candidates
    text = export_wisdom()          # JSON, for a file
    import_wisdom(text)             # in a later process, before planning
    forget_wisdom()                 # back to the built-in defaults
    set_l2_block_bytes(1 << 20)     # smaller L2 blocks for plans created next

Settings are process-wide per (precision, length): plans created after a
tune or an import use them; plans created before keep theirs.
"""
import ctypes
import json

from ._lib import GOFFT_C2C, GOFFT_F32, GOFFT_F32MIXED, GOFFT_F64, GOFFT_R2C, GoFFTError, check, last_error, lib

_PREC = {"f64": GOFFT_F64, "f32": GOFFT_F32, "f32mixed": GOFFT_F32MIXED}
_KIND = {"c2c": GOFFT_C2C, "r2c": GOFFT_R2C}


def _text(n_or_status, fill):
    if n_or_status < 0:
        raise GoFFTError(-n_or_status, last_error())
    buf = ctypes.create_string_buffer(int(n_or_status) + 1)
    fill(buf, n_or_status + 1)
    return buf.value.decode()


def autotune(kind, precision, shape, batch=1):
    """Tunes batched transforms of `shape`; returns the wisdom as a dict."""
    k = _KIND[kind] if isinstance(kind, str) else int(kind)
    p = _PREC[precision] if isinstance(precision, str) else int(precision)
    sh = (ctypes.c_int64 * len(shape))(*[int(s) for s in shape])
    n = lib().gofft_autotune(k, p, sh, len(shape), int(batch), None, 0)
    return json.loads(_text(n, lambda b, c: lib().gofft_wisdom_export(b, c)))


def autotune_uneven(precision, lengths):
    """Tunes the schedule of each length class of an uneven batch."""
    p = _PREC[precision] if isinstance(precision, str) else int(precision)
    arr = (ctypes.c_int64 * len(lengths))(*[int(v) for v in lengths])
    n = lib().gofft_autotune_uneven(p, arr, len(lengths), None, 0)
    return json.loads(_text(n, lambda b, c: lib().gofft_wisdom_export(b, c)))


def export_wisdom():
    n = lib().gofft_wisdom_export(None, 0)
    return _text(n, lambda b, c: lib().gofft_wisdom_export(b, c))


def import_wisdom(text):
    if isinstance(text, dict):
        text = json.dumps(text)
    check(lib().gofft_wisdom_import(text.encode()))


def forget_wisdom():
    check(lib().gofft_wisdom_forget())


def set_l2_block_bytes(nbytes):
    """Complex intermediate bytes per L2 block for plans created afterwards
    (rank-2 real plans: images per block; complex N-D plans: planes per
    block); nbytes <= 0 restores the default of 48 MiB."""
    check(lib().gofft_set_l2_block_bytes(int(nbytes)))


def set_lanes(lanes):
    """Streams plans created afterwards rotate their L2 blocks over: 2 (the
    default; 0 restores it) or 1 (blocks back to back, each pass alone)."""
    check(lib().gofft_set_lanes(int(lanes)))


def set_tma_pipeline(on):
    """The TMA-fed persistent line kernel on or off (the default) for
    launches made afterwards (results agree to rounding; a comparison
    switch)."""
    check(lib().gofft_set_tma_pipeline(1 if on else 0))


def set_dependent_launch(mode):
    """Programmatic dependent launch of the line kernels made afterwards:
    0 off, 1 each waits on the device for its predecessor, 2 also lets the
    next one be scheduled early (results identical in every mode)."""
    check(lib().gofft_set_dependent_launch(int(mode)))


def pipeline_status():
    """Raises if a pipelined line kernel's bounded wait gave up since the
    last call (synchronises the device)."""
    check(lib().gofft_pipeline_status())
