package gofftcuda

/*
#include "gofft.h"
*/
import "C"

// Spectral helpers (freq.go:17-127, window.go:20-100).

// FFTFreq returns the n sample frequencies of FFT bins at spacing d
// (freq.go:17-37).
func FFTFreq(n int, d float64) []float64 {
	if n <= 0 {
		return []float64{}
	}
	out := make([]float64, n)
	check(C.gofft_fftfreq(C.int64_t(n), C.double(d), reals(out)))
	return out
}

// RFFTFreq returns the n/2+1 frequencies of RFFT bins (freq.go:45-56).
func RFFTFreq(n int, d float64) []float64 {
	if n <= 0 {
		return []float64{}
	}
	out := make([]float64, n/2+1)
	check(C.gofft_rfftfreq(C.int64_t(n), C.double(d), reals(out)))
	return out
}

// PSD returns the one-sided power spectral density of x (freq.go:69-90).
func PSD(x []float64, d float64) []float64 {
	if len(x) == 0 {
		return []float64{}
	}
	out := make([]float64, len(x)/2+1)
	check(C.gofft_psd(reals(x), C.int64_t(len(x)), C.double(d), reals(out)))
	return out
}

// Spectrogram returns the PSD of each windowed frame (freq.go:107-127); it
// panics on the reference's bad arguments.  Even segments run as one fused
// device launch over all frames.
func Spectrogram(x []float64, segment, overlap int, window []float64, d float64) [][]float64 {
	var nf C.int64_t
	check(C.gofft_spectrogram(reals(x), C.int64_t(len(x)), C.int64_t(segment), C.int64_t(overlap), reals(window),
		C.int64_t(len(window)), C.double(d), nil, &nf))
	if nf == 0 {
		return nil
	}
	bins := segment/2 + 1
	flat := make([]float64, int(nf)*bins)
	check(C.gofft_spectrogram(reals(x), C.int64_t(len(x)), C.int64_t(segment), C.int64_t(overlap), reals(window),
		C.int64_t(len(window)), C.double(d), reals(flat), &nf))
	frames := make([][]float64, int(nf))
	for t := range frames {
		frames[t] = flat[t*bins : (t+1)*bins : (t+1)*bins]
	}
	return frames
}

func window(n int, f func(C.int64_t, *C.double) C.int) []float64 {
	if n <= 0 {
		return []float64{}
	}
	out := make([]float64, n)
	check(f(C.int64_t(n), reals(out)))
	return out
}

// Hann returns the symmetric Hann window (window.go:20-22).
func Hann(n int) []float64 {
	return window(n, func(m C.int64_t, p *C.double) C.int { return C.gofft_hann(m, p) })
}

// Hamming returns the symmetric Hamming window (window.go:29-31).
func Hamming(n int) []float64 {
	return window(n, func(m C.int64_t, p *C.double) C.int { return C.gofft_hamming(m, p) })
}

// Blackman returns the symmetric Blackman window (window.go:38-40).
func Blackman(n int) []float64 {
	return window(n, func(m C.int64_t, p *C.double) C.int { return C.gofft_blackman(m, p) })
}

// BlackmanHarris returns the symmetric 4-term Blackman-Harris window
// (window.go:48-50).
func BlackmanHarris(n int) []float64 {
	return window(n, func(m C.int64_t, p *C.double) C.int { return C.gofft_blackman_harris(m, p) })
}

// Bartlett returns the symmetric triangular window (window.go:86-100).
func Bartlett(n int) []float64 {
	return window(n, func(m C.int64_t, p *C.double) C.int { return C.gofft_bartlett(m, p) })
}
