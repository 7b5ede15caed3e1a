package gofftcuda

/*
#include "gofft.h"
*/
import "C"

// The N-D and 2-D transforms (ndfft.go:22-62, rfft2.go:22-138): one device
// call per transform (every axis runs on the GPU; the reference's goroutine
// fan-out over lines, parallel.go:32-61, is the grid of a launch).

func validateShape(shape []int, total int) {
	prod := 1
	for _, s := range shape {
		if s <= 0 {
			panic("fft: shape lengths must be positive")
		}
		prod *= s
	}
	if prod != total {
		panic("fft: shape product does not match len(data)")
	}
}

func transformN(data []complex128, shape []int, inverse bool) []complex128 {
	validateShape(shape, len(data))
	out := make([]complex128, len(data))
	if len(data) <= 1 {
		copy(out, data)
		return out
	}
	sh := make([]C.int64_t, len(shape))
	for i, s := range shape {
		sh[i] = C.int64_t(s)
	}
	if inverse {
		check(C.gofft_ifftn(cplx(data), C.int64_t(len(data)), &sh[0], C.int(len(shape)), cplx(out)))
	} else {
		check(C.gofft_fftn(cplx(data), C.int64_t(len(data)), &sh[0], C.int(len(shape)), cplx(out)))
	}
	return out
}

// FFTN is the forward N-dimensional DFT of row-major data (ndfft.go:22-24).
func FFTN(data []complex128, shape []int) []complex128 { return transformN(data, shape, false) }

// IFFTN is its normalised inverse (ndfft.go:31-33).
func IFFTN(data []complex128, shape []int) []complex128 { return transformN(data, shape, true) }

// FFT2 is the 2-D FFTN (ndfft.go:37-39).
func FFT2(data []complex128, shape [2]int) []complex128 { return FFTN(data, shape[:]) }

// IFFT2 is the 2-D IFFTN (ndfft.go:43-45).
func IFFT2(data []complex128, shape [2]int) []complex128 { return IFFTN(data, shape[:]) }

// RFFT2 returns the shape[0] x (shape[1]/2+1) half spectrum of a real
// row-major matrix (rfft2.go:22-74).
func RFFT2(data []float64, shape [2]int) []complex128 {
	rows, cols := shape[0], shape[1]
	if rows <= 0 || cols <= 0 {
		panic("fft: shape lengths must be positive")
	}
	if rows*cols != len(data) {
		panic("fft: shape product does not match len(data)")
	}
	out := make([]complex128, rows*(cols/2+1))
	check(C.gofft_rfft2(reals(data), C.int64_t(len(data)), C.int64_t(rows), C.int64_t(cols), cplx(out)))
	return out
}

// IRFFT2 inverts RFFT2; bins beyond len(data) read as zero (rfft2.go:87-138).
func IRFFT2(data []complex128, shape [2]int) []float64 {
	rows, cols := shape[0], shape[1]
	if rows <= 0 || cols <= 0 {
		panic("fft: shape lengths must be positive")
	}
	out := make([]float64, rows*cols)
	check(C.gofft_irfft2(cplx(data), C.int64_t(len(data)), C.int64_t(rows), C.int64_t(cols), reals(out)))
	return out
}
