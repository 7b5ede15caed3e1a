/*
 * gofft_oracle.h -- CPU restatement of go-fft/fft's transform path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA engine is
 * compared against (tests/, __graft_entry__.smoke(), and bench.py's
 * cpu_baseline / --impl reference leg).  Nothing in the product path links or
 * calls it.
 *
 * Every routine restates the reference algorithm in plain C99 with the same
 * evaluation order: complex products are written as explicit real formulas
 * (ar*br - ai*bi, ar*bi + ai*br), and the file is compiled with
 * -ffp-contract=off so no multiply-add is fused, matching Go on amd64
 * (GOAMD64=v1), which never fuses.  Twiddles come from glibc cos/sin, which
 * can differ from Go's pure-Go math.Cos/Sin by about one ulp, so results are
 * not bitwise equal to Go but agree far inside 1e-12; integer tables are
 * bit-exact by construction.
 */
#ifndef GOFFT_ORACLE_H
#define GOFFT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Engine selected by the reference router NewPlan (plan.go:42-73). */
enum { OR_TRIVIAL = 0, OR_IT = 1, OR_CT = 2, OR_RADER = 3, OR_BLUESTEIN = 4 };

/* --- integer helpers (plan.go, rader.go, iterative.go, bluestein.go) ----- */
int  or_engine(int n);                                  /* plan.go:42-73 */
int  or_factors_small(int n);                           /* plan.go:134 */
int  or_factorize(int n, int *out);                     /* plan.go:265; returns count */
int  or_next_smooth_conv(int lo);                       /* plan.go:154 */
int  or_conv_cost(int m, double *cost);                 /* plan.go:192; returns ok */
int  or_best_conv_len(int lo);                          /* plan.go:241 */
int  or_is_prime(int n);                                /* rader.go:232 */
int  or_primitive_root(int p);                          /* rader.go:178 */
int  or_it_radices(int n, int *out);                    /* iterative.go:59-80 */
void or_rev_pos(int n, int *out);                       /* iterative.go:87-103 */
void or_bit_reverse_perm(int n, int *out);              /* kernels.go:20-32 as a permutation */
/* Rader tables (rader.go:51-91): returns cl, writes cyclic flag, generator,
 * perm[q] and iperm[q] (q = n-1). */
int  or_rader_info(int n, int *cyclic, int *g, int *perm, int *iperm);
/* Bluestein chirp index j*j mod 2n (bluestein.go:38) and conv length m. */
int  or_bluestein_m(int n);
void or_chirp_index(int n, int64_t *out);

/* --- complex transforms (complex128 interleaved re,im) ------------------- */
/* Plan.FFT / Plan.IFFT through the plan cache (plan.go:91-109, 301-317).
 * dst may alias src. */
void or_fft(int n, double *dst, const double *src);
void or_ifft(int n, double *dst, const double *src);
/* Unnormalised engine call Plan.execute (plan.go:113-129). */
void or_execute(int n, double *dst, const double *src, int inverse);
/* Bluestein / Rader engines built directly (tests cross-check them). */
void or_bluestein_transform(int n, double *dst, const double *src, int inverse);
void or_rader_transform(int n, double *dst, const double *src, int inverse);

/* --- real transforms (realplan.go, rfft.go) ------------------------------ */
void or_rfft(int n, double *dst /* n/2+1 complex */, const double *src /* n */);
void or_irfft(int n, double *dst /* n */, const double *src, int nsrc /* bins */);

/* --- 2-D / N-D (rfft2.go, ndfft.go, parallel.go) ------------------------- */
void or_set_workers(int w);                             /* parallel.go:18 */
int  or_get_workers(void);
void or_fftn(double *out, const double *data, const int *shape, int rank, int inverse);
void or_rfft2(double *out /* rows*(cols/2+1) complex */, const double *data, int rows, int cols);
void or_irfft2(double *out /* rows*cols */, const double *data, int64_t ndata /* complex count */,
               int rows, int cols);

/* --- spectral helpers (freq.go, window.go) ------------------------------- */
void or_cosine_window(int n, const double *a, int na, double *out);   /* window.go:59-78 */
void or_hann(int n, double *out);                                     /* window.go:20-22 */
void or_psd(int n, const double *x, double d, double *out);           /* freq.go:69-90 */
/* Spectrogram (freq.go:107-127): returns frame count; out holds
 * frames*(segment/2+1) values when non-NULL. */
int  or_spectrogram(const double *x, int64_t nx, int segment, int overlap,
                    const double *window, double d, double *out);

/* --- batch helper for the CPU baseline: `batch` independent Plan.FFT (or
 * IFFT) calls split across the worker pool with parChunks chunking. ------- */
void or_batch_fft(int n, int64_t batch, double *dst, const double *src, int inverse);
void or_batch_rfft2_roundtrip(int64_t batch, int rows, int cols, const double *x,
                              double *spec, double *back);

#ifdef __cplusplus
}
#endif
#endif
