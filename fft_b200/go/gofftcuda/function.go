package gofftcuda

/*
#include "gofft.h"
*/
import "C"

import "unsafe"

// Function is one differentiable step on device buffers, mirroring
// torch.autograd.Function: Forward computes (and saves what Backward needs),
// Backward maps output gradients to input gradients (vector-Jacobian
// products, real inner product Re sum conj(a) b).  No counterpart in the
// reference, which has no differentiation.  The buffers are device pointers
// from the caller's CUDA allocator; stream may be nil (the default stream).
type Function interface {
	Forward(in, out unsafe.Pointer)
	Backward(gradOut, gradIn unsafe.Pointer)
}

// DevicePlan is a batched device-resident plan (gofft_plan_create).
type DevicePlan struct {
	h      *C.gofft_plan
	stream C.gofft_stream
}

// Precision of a device plan.
const (
	F64      = C.GOFFT_F64      // complex128 / float64
	F32      = C.GOFFT_F32      // complex64, twiddles rounded once
	F32Mixed = C.GOFFT_F32MIXED // complex64, FP64-derived hi+lo twiddles
)

// NewDevicePlan creates a plan of kind C2C (complex) or R2C (real) over
// `batch` contiguous transforms of `shape`.
func NewDevicePlan(isReal bool, precision int, shape []int, batch int) *DevicePlan {
	kind := C.int(C.GOFFT_C2C)
	if isReal {
		kind = C.GOFFT_R2C
	}
	sh := make([]C.int64_t, len(shape))
	for i, s := range shape {
		sh[i] = C.int64_t(s)
	}
	var h *C.gofft_plan
	check(C.gofft_plan_create(kind, C.int(precision), &sh[0], C.int(len(shape)), C.int64_t(batch), 0, 0, 0, 0, &h))
	return &DevicePlan{h: h}
}

// Close releases the plan.
func (p *DevicePlan) Close() { C.gofft_plan_destroy(p.h) }

// FFTFunc is the batched complex FFT (inverse: the normalised IFFT).
type FFTFunc struct {
	Plan    *DevicePlan
	Inverse bool
}

func b2i(b bool) C.int {
	if b {
		return 1
	}
	return 0
}

func (f *FFTFunc) Forward(in, out unsafe.Pointer) {
	check(C.gofft_exec_c2c(f.Plan.h, in, out, b2i(f.Inverse), f.Plan.stream))
}
func (f *FFTFunc) Backward(g, gin unsafe.Pointer) {
	check(C.gofft_vjp_c2c(f.Plan.h, g, gin, b2i(f.Inverse), f.Plan.stream))
}

// RFFTFunc is the batched real forward (RFFT, or RFFT2 for a rank-2 plan).
type RFFTFunc struct{ Plan *DevicePlan }

func (f *RFFTFunc) Forward(in, out unsafe.Pointer) {
	check(C.gofft_exec_r2c(f.Plan.h, in, out, f.Plan.stream))
}
func (f *RFFTFunc) Backward(g, gin unsafe.Pointer) {
	check(C.gofft_vjp_r2c(f.Plan.h, g, gin, f.Plan.stream))
}

// IRFFTFunc is the batched real inverse (IRFFT, or IRFFT2 for a rank-2 plan).
type IRFFTFunc struct{ Plan *DevicePlan }

func (f *IRFFTFunc) Forward(in, out unsafe.Pointer) {
	check(C.gofft_exec_c2r(f.Plan.h, in, 0, out, f.Plan.stream))
}
func (f *IRFFTFunc) Backward(g, gin unsafe.Pointer) {
	check(C.gofft_vjp_c2r(f.Plan.h, g, gin, f.Plan.stream))
}

// SpectralFilter2 is y = IRFFT2(H * RFFT2(x)) over a batch of images (a
// rank-2 real plan).  Forward saves the spectra RFFT2(x) in Saved (batch *
// rows * (cols/2+1) complex, device) for Backward's dH; Backward writes dx
// into gradIn and dH into DH.  Passing Saved as the scratch lets Backward
// overwrite it (one Backward per Forward).
type SpectralFilter2 struct {
	Plan  *DevicePlan
	H     unsafe.Pointer // rows * (cols/2+1) complex
	Saved unsafe.Pointer
	DH    unsafe.Pointer
}

func (f *SpectralFilter2) Forward(x, y unsafe.Pointer) {
	check(C.gofft_filter2_forward(f.Plan.h, x, f.H, y, f.Saved, f.Plan.stream))
}
func (f *SpectralFilter2) Backward(g, dx unsafe.Pointer) {
	check(C.gofft_vjp_filter2(f.Plan.h, g, f.H, f.Saved, f.Saved, dx, f.DH, f.Plan.stream))
}
