// Package gofftcuda is go-fft/fft's public API on the B200 engine
// (libgofft_b200.so, C-ABI in include/gofft.h), through cgo.  Every function
// keeps the reference's signature and semantics: inputs are never modified,
// results are newly allocated, empty input returns an empty non-nil slice,
// length 1 returns a copy, inverses are normalised, and bad shapes or
// spectrogram arguments panic with the reference's messages.  A program
// switches by importing this package under the name fft.
//
// Host buffers are passed to the engine for the duration of one call only
// (the engine copies them to and from the device inside the call), so no Go
// pointer is retained and cgo's pointer rules hold.  []complex128 is passed
// as interleaved (re, im) float64 pairs, its memory layout.
//
// Reference files: fft.go:14-51 (FFT, IFFT, FFTReal), plan.go:42-109
// (NewPlan, Plan), realplan.go:37-192 (NewRealPlan, RealPlan), rfft.go:19-45
// (RFFT, IRFFT), rfft2.go:22-138 (RFFT2, IRFFT2), ndfft.go:22-62 (FFTN,
// IFFTN, FFT2, IFFT2), freq.go:17-127 (FFTFreq, RFFTFreq, PSD, Spectrogram),
// window.go:20-100 (windows).
package gofftcuda

/*
#cgo CFLAGS: -I${SRCDIR}/../../../include
#cgo LDFLAGS: -L${SRCDIR}/../.. -lgofft_b200 -Wl,-rpath,${SRCDIR}/../..
#include <stdlib.h>
#include "gofft.h"
*/
import "C"

import "unsafe"

func check(st C.int) {
	if st != C.GOFFT_OK {
		panic(C.GoString(C.gofft_last_error()))
	}
}

func cplx(s []complex128) *C.double {
	if len(s) == 0 {
		return nil
	}
	return (*C.double)(unsafe.Pointer(&s[0]))
}

func reals(s []float64) *C.double {
	if len(s) == 0 {
		return nil
	}
	return (*C.double)(unsafe.Pointer(&s[0]))
}

// FFT returns the forward DFT of x (fft.go:14-23).
func FFT(x []complex128) []complex128 {
	out := make([]complex128, len(x))
	if len(x) <= 1 {
		copy(out, x)
		return out
	}
	check(C.gofft_fft(cplx(x), C.int64_t(len(x)), cplx(out)))
	return out
}

// IFFT returns the inverse DFT of x, normalised by N (fft.go:31-40).
func IFFT(x []complex128) []complex128 {
	out := make([]complex128, len(x))
	if len(x) <= 1 {
		copy(out, x)
		return out
	}
	check(C.gofft_ifft(cplx(x), C.int64_t(len(x)), cplx(out)))
	return out
}

// FFTReal returns the full complex spectrum of a real signal (fft.go:45-51).
func FFTReal(x []float64) []complex128 {
	c := make([]complex128, len(x))
	for i, v := range x {
		c[i] = complex(v, 0)
	}
	return FFT(c)
}

// Plan is a complex transform of one length (plan.go:19-30); safe for
// concurrent use.
type Plan struct {
	h *C.gofft_plan
	n int
}

// NewPlan builds a plan for length n (plan.go:42-73); n <= 1 gives the
// trivial plan.
func NewPlan(n int) *Plan {
	if n < 0 {
		return &Plan{n: n}
	}
	var h *C.gofft_plan
	check(C.gofft_new_plan(C.int64_t(n), &h))
	return &Plan{h: h, n: n}
}

// Len reports the plan's length (plan.go:86).
func (p *Plan) Len() int { return p.n }

// FFT writes the forward DFT of src into dst and returns dst; dst may alias
// src (plan.go:91-94).
func (p *Plan) FFT(dst, src []complex128) []complex128 {
	if p.n <= 0 {
		return dst
	}
	check(C.gofft_plan_fft(p.h, cplx(dst), cplx(src)))
	return dst
}

// IFFT writes the inverse DFT of src (normalised by N) into dst and returns
// dst (plan.go:98-109).
func (p *Plan) IFFT(dst, src []complex128) []complex128 {
	if p.n <= 0 {
		return dst
	}
	check(C.gofft_plan_ifft(p.h, cplx(dst), cplx(src)))
	return dst
}

// RealPlan is a real transform of one length (realplan.go:17-33).
type RealPlan struct {
	h *C.gofft_plan
	n int
}

// NewRealPlan builds a real plan for length n (realplan.go:37-58).
func NewRealPlan(n int) *RealPlan {
	if n < 0 {
		return &RealPlan{n: n}
	}
	var h *C.gofft_plan
	check(C.gofft_new_real_plan(C.int64_t(n), &h))
	return &RealPlan{h: h, n: n}
}

// Len reports the real-input length (realplan.go:72).
func (p *RealPlan) Len() int { return p.n }

// RFFT writes the N/2+1 bins of src into dst and returns dst[:N/2+1]
// (realplan.go:77-116).
func (p *RealPlan) RFFT(dst []complex128, src []float64) []complex128 {
	if p.n <= 0 {
		return dst[:0]
	}
	check(C.gofft_real_plan_rfft(p.h, cplx(dst), reals(src)))
	return dst[:p.n/2+1]
}

// IRFFT reconstructs the length-N real signal from up to N/2+1 bins of src
// (missing bins read as zero), normalised by N (realplan.go:181-192).
func (p *RealPlan) IRFFT(dst []float64, src []complex128) []float64 {
	if p.n <= 0 {
		return dst[:0]
	}
	check(C.gofft_real_plan_irfft(p.h, reals(dst), cplx(src), C.int64_t(len(src))))
	return dst[:p.n]
}

// RFFT returns the non-redundant half spectrum of x (rfft.go:19-26).
func RFFT(x []float64) []complex128 {
	if len(x) == 0 {
		return []complex128{}
	}
	out := make([]complex128, len(x)/2+1)
	check(C.gofft_rfft(reals(x), C.int64_t(len(x)), cplx(out)))
	return out
}

// IRFFT inverts RFFT for output length n (rfft.go:39-45).
func IRFFT(spectrum []complex128, n int) []float64 {
	if n <= 0 {
		return []float64{}
	}
	out := make([]float64, n)
	check(C.gofft_irfft(cplx(spectrum), C.int64_t(len(spectrum)), C.int64_t(n), reals(out)))
	return out
}
