"""fft_b200 -- a B200-native engine for go-fft/fft's transform path.

The product is libgofft_b200.so (CUDA for sm_100a behind the C-ABI in
include/gofft.h).  This package loads it and exposes:

* ``fft_b200.gofft`` -- the reference's Go API, call for call (NewPlan,
  Plan.FFT/IFFT, NewRealPlan, RFFT/IRFFT, FFT2/IFFT2, FFTN/IFFTN,
  RFFT2/IRFFT2, PSD, Spectrogram, Hann) on numpy arrays;
* ``fft_b200.device`` -- batched device-resident plans on torch tensors in
  FP64 and the FP32 forms.
"""
from ._lib import LIB_PATH, GoFFTError, lib  # noqa: F401

__all__ = ["lib", "LIB_PATH", "GoFFTError"]
