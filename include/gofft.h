/*
 * gofft.h -- C-ABI of the B200 FFT engine (libgofft_b200.so).
 *
 * The engine is a drop-in for the transform path of go-fft/fft.  Two layers:
 *
 *  1. The reference-facing entry points (gofft_new_plan ... gofft_spectrogram)
 *     mirror the Go API one call for one call: host buffers of complex128
 *     (interleaved re,im doubles) or float64, one transform per call, the same
 *     argument meaning and normalisation.  A cgo binding calls these.
 *     Argument errors that the Go API turns into a panic
 *     return GOFFT_EINVAL with the reference's panic text in
 *     gofft_last_error().
 *
 *  2. Device-resident plans (gofft_plan_create / gofft_exec_*) for batched,
 *     strided transforms on device pointers in FP64 or the FP32 forms, plus
 *     host-pointer variants that copy in and out inside the call.
 *
 * Every function returns a gofft_status; none aborts.  Plans are immutable
 * after creation.  A plan's workspace is shared by its executions, so
 * executions of one plan must not overlap on the device; the host-pointer and
 * reference-facing entry points serialise on a per-plan lock.
 */
#ifndef GOFFT_H
#define GOFFT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GOFFT_API __attribute__((visibility("default")))
#else
#define GOFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gofft_plan gofft_plan;
typedef void *gofft_stream; /* a cudaStream_t; NULL = legacy default stream */

typedef enum {
  GOFFT_OK = 0,
  GOFFT_EINVAL = 1,       /* invalid argument (reference: panic) */
  GOFFT_ENOMEM = 2,       /* device allocation failed */
  GOFFT_ECUDA = 3,        /* CUDA runtime error */
  GOFFT_ETIMEOUT = 4,     /* a bounded device wait expired */
  GOFFT_EUNSUPPORTED = 5  /* shape/layout not supported by this build */
} gofft_status;

typedef enum {
  GOFFT_C2C = 0, /* complex <-> complex */
  GOFFT_R2C = 1  /* real forward (R2C) and its inverse (C2R); last axis real */
} gofft_kind;

typedef enum {
  GOFFT_F64 = 0,      /* complex128 / float64: the parity form */
  GOFFT_F32 = 1,      /* complex64, FP64-generated twiddles rounded to FP32 */
  GOFFT_F32MIXED = 2  /* complex64, FP64 twiddles as hi+lo FP32 pairs */
} gofft_precision;

/* Last error message of the calling thread ("" if none). */
GOFFT_API const char *gofft_last_error(void);
/* Library version string. */
GOFFT_API const char *gofft_version(void);

/* ------------------------------------------------------------------------ */
/* 1. Reference-facing entry points (FP64, host buffers, one call each).     */
/* ------------------------------------------------------------------------ */

/* NewPlan (plan.go:42-73): a plan for length n >= 0; serves FFT and IFFT. */
GOFFT_API int gofft_new_plan(int64_t n, gofft_plan **out);
/* cachedPlan (plan.go:301-317): the shared memoised plan for n (not owned by
 * the caller; never destroy it). */
GOFFT_API int gofft_cached_plan(int64_t n, gofft_plan **out);
/* Plan.Len (plan.go:86). */
GOFFT_API int64_t gofft_plan_len(const gofft_plan *p);
/* Plan.FFT (plan.go:91-94): dst, src hold Len() complex128; dst may alias. */
GOFFT_API int gofft_plan_fft(gofft_plan *p, double *dst, const double *src);
/* Plan.IFFT (plan.go:98-109): inverse normalised by 1/N; dst may alias. */
GOFFT_API int gofft_plan_ifft(gofft_plan *p, double *dst, const double *src);

/* NewRealPlan (realplan.go:37-58). */
GOFFT_API int gofft_new_real_plan(int64_t n, gofft_plan **out);
/* RealPlan.RFFT (realplan.go:77-116): src n float64 -> dst n/2+1 complex128. */
GOFFT_API int gofft_real_plan_rfft(gofft_plan *p, double *dst, const double *src);
/* RealPlan.IRFFT (realplan.go:181-192): reads min(nsrc, n/2+1) bins (missing
 * bins are zero, imaginary parts of DC/Nyquist ignored); writes n float64
 * normalised by 1/n. */
GOFFT_API int gofft_real_plan_irfft(gofft_plan *p, double *dst, const double *src, int64_t nsrc);

/* FFT / IFFT / FFTReal (fft.go:14-51): out has n complex128. */
GOFFT_API int gofft_fft(const double *x, int64_t n, double *out);
GOFFT_API int gofft_ifft(const double *x, int64_t n, double *out);
GOFFT_API int gofft_fft_real(const double *x, int64_t n, double *out);
/* RFFT (rfft.go:19-26): out has n/2+1 complex128 (0 for n == 0). */
GOFFT_API int gofft_rfft(const double *x, int64_t n, double *out);
/* IRFFT (rfft.go:39-45): spectrum of nspec bins -> n float64 (n <= 0: none). */
GOFFT_API int gofft_irfft(const double *spectrum, int64_t nspec, int64_t n, double *out);

/* FFTN / IFFTN (ndfft.go:22-33): data of len complex128, row-major shape of
 * rank dims (rank 0 = scalar).  EINVAL ("fft: shape lengths must be
 * positive" / "fft: shape product does not match len(data)") where the
 * reference panics.  out has len complex128. */
GOFFT_API int gofft_fftn(const double *data, int64_t len, const int64_t *shape, int rank, double *out);
GOFFT_API int gofft_ifftn(const double *data, int64_t len, const int64_t *shape, int rank, double *out);
/* FFT2 / IFFT2 (ndfft.go:37-45). */
GOFFT_API int gofft_fft2(const double *data, int64_t len, int64_t rows, int64_t cols, double *out);
GOFFT_API int gofft_ifft2(const double *data, int64_t len, int64_t rows, int64_t cols, double *out);
/* RFFT2 (rfft2.go:22-74): rows*cols float64 -> rows*(cols/2+1) complex128. */
GOFFT_API int gofft_rfft2(const double *data, int64_t len, int64_t rows, int64_t cols, double *out);
/* IRFFT2 (rfft2.go:87-138): reads up to rows*(cols/2+1) bins of len (the rest
 * zero) -> rows*cols float64 normalised by 1/(rows*cols). */
GOFFT_API int gofft_irfft2(const double *data, int64_t len, int64_t rows, int64_t cols, double *out);

/* Hann (window.go:20-22): symmetric window of length n (n <= 0: none). */
GOFFT_API int gofft_hann(int64_t n, double *out);
/* Hamming, Blackman, BlackmanHarris, Bartlett (window.go:29-100): symmetric
 * windows of length n (n <= 0: none, n == 1: {1}). */
GOFFT_API int gofft_hamming(int64_t n, double *out);
GOFFT_API int gofft_blackman(int64_t n, double *out);
GOFFT_API int gofft_blackman_harris(int64_t n, double *out);
GOFFT_API int gofft_bartlett(int64_t n, double *out);
/* FFTFreq (freq.go:17-37): n bin frequencies for spacing d; RFFTFreq
 * (freq.go:46-56): n/2+1 of them (n <= 0: none). */
GOFFT_API int gofft_fftfreq(int64_t n, double d, double *out);
GOFFT_API int gofft_rfftfreq(int64_t n, double d, double *out);
/* PSD (freq.go:69-90): one-sided density of n reals at spacing d -> n/2+1. */
GOFFT_API int gofft_psd(const double *x, int64_t n, double d, double *out);
/* Spectrogram (freq.go:107-127): frames of `segment` samples every
 * segment-overlap samples, windowed, PSD each.  *nframes receives the frame
 * count; out (frames*(segment/2+1) float64) may be NULL to query it. */
GOFFT_API int gofft_spectrogram(const double *x, int64_t nx, int64_t segment, int64_t overlap,
                      const double *window, int64_t nwindow, double d, double *out,
                      int64_t *nframes);

/* ------------------------------------------------------------------------ */
/* 2. Device-resident plans.                                                 */
/* ------------------------------------------------------------------------ */

/* Plan for `batch` transforms of a row-major `shape` (rank >= 1).
 *  C2C: element i (flattened index) of transform b is at b*idist + i*istride
 *       (rank 1 any strides; rank > 1 requires istride == ostride == 1).
 *  R2C: the last axis is real of length shape[rank-1] = n; the complex side
 *       has n/2+1 bins on that axis.  "in" is the real side for strides and
 *       distances (idist/istride in reals, odist/ostride in complex bins);
 *       rank is 1 or 2.
 * Strides/distances of 0 select the contiguous defaults. */
GOFFT_API int gofft_plan_create(int kind, int precision, const int64_t *shape, int rank, int64_t batch,
                      int64_t istride, int64_t idist, int64_t ostride, int64_t odist,
                      gofft_plan **out);
GOFFT_API int gofft_plan_destroy(gofft_plan *p);
/* Bytes of device workspace the plan owns. */
GOFFT_API int gofft_plan_workspace_size(const gofft_plan *p, size_t *bytes);
/* JSON description of the plan (engine per axis, radix schedule, launch
 * shape); returns the full length, writes at most cap bytes. */
GOFFT_API int64_t gofft_plan_describe(const gofft_plan *p, char *buf, int64_t cap);

/* Forward (inverse = 0) or normalised inverse (inverse = 1) C2C on device
 * pointers.  in == out is allowed. */
GOFFT_API int gofft_exec_c2c(gofft_plan *p, const void *in, void *out, int inverse, gofft_stream stream);
/* R2C on device pointers (real in, complex out). */
GOFFT_API int gofft_exec_r2c(gofft_plan *p, const void *in, void *out, gofft_stream stream);
/* C2R on device pointers: nbins complex bins per last-axis line are read
 * (nbins <= 0 means n/2+1); output normalised by 1/prod(shape). */
GOFFT_API int gofft_exec_c2r(gofft_plan *p, const void *in, int64_t nbins, void *out, gofft_stream stream);

/* gofft_exec_c2c for a 1-D complex plan without allocating anything (no
 * counterpart in the reference, whose transforms allocate per call).  For
 * callers that cannot have device memory allocated while they run -- work
 * being recorded into a CUDA graph, device memory owned by another allocator's
 * budget, or paths that cannot afford cudaMalloc's device-wide
 * synchronisation.  Scratch comes from one 16 MiB array built into the
 * library (held on every GPU that loads it); transforms needing more return
 * GOFFT_EINVAL, a plan that is not complex-to-complex GOFFT_EINVAL, and a
 * complex plan of rank above 1 GOFFT_EUNSUPPORTED.  The first call on a device
 * looks the array up and should come before any stream capture.  All calls
 * share the array: calls whose executions overlap on the GPU race and must be
 * serialised by the caller. */
GOFFT_API int gofft_exec_c2c_noalloc(gofft_plan *p, const void *in, void *out, int inverse,
                                     gofft_stream stream);

/* Host-pointer variants: copy host -> device, execute, copy back, synchronise.
 * Pinned host memory makes the copies asynchronous DMA.  Batched 2-D real
 * plans (r2c / c2r) pipeline the batch in blocks of images: one block copies
 * in while the previous one transforms and the one before copies out, so both
 * PCIe directions overlap (rfft2.go:22-138 is the per-call reference path). */
GOFFT_API int gofft_exec_c2c_host(gofft_plan *p, const void *in, void *out, int inverse);
GOFFT_API int gofft_exec_r2c_host(gofft_plan *p, const void *in, void *out);
GOFFT_API int gofft_exec_c2r_host(gofft_plan *p, const void *in, int64_t nbins, void *out);

/* Integer tables of a 1-D plan (bit-exact with the reference):
 * which = 0: Rader perm[k] = g^k mod p (rader.go:67-70), 1: Rader iperm,
 * 2: Bluestein chirp index j*j mod 2n (bluestein.go:38), 3: Rader generator
 * g and convolution length (2 values), 4: Bluestein convolution length m.
 * Returns the table length (or -1 if the plan has no such table); copies at
 * most cap entries. */
GOFFT_API int64_t gofft_plan_table(const gofft_plan *p, int which, int64_t *out, int64_t cap);

/* Spectrogram on device buffers in any precision (real type per precision):
 * x has nx samples, window `segment` samples; out receives
 * frames*(segment/2+1) densities; segment must be even. */
GOFFT_API int gofft_spectrogram_device(int precision, const void *x, int64_t nx, int64_t segment,
                             int64_t overlap, const void *window, double d, void *out,
                             int64_t *nframes, gofft_stream stream);

/* A window (kind 0 Hann, 1 Hamming, 2 Blackman, 3 Blackman-Harris,
 * 4 Bartlett; window.go:20-100) of n samples generated on the device in FP64
 * (angles from exact integer residues) and stored in the precision's real
 * type.  No reference counterpart (the reference builds windows on the host). */
GOFFT_API int gofft_window_device(int precision, int kind, int64_t n, void *out, gofft_stream stream);
/* gofft_spectrogram_device with a window of `window_kind` generated on the
 * device (once per kind, length and precision, then kept) instead of a
 * caller's buffer. */
GOFFT_API int gofft_spectrogram_window_device(int precision, const void *x, int64_t nx, int64_t segment,
                                              int64_t overlap, int window_kind, double d, void *out,
                                              int64_t *nframes, gofft_stream stream);

/* ------------------------------------------------------------------------ */
/* 2b. Uneven batches (no counterpart in the reference, whose batches are a   */
/*     caller loop over Plan.FFT, plan.go:91): many complex transforms of     */
/*     different lengths in one persistent launch.                            */
/* ------------------------------------------------------------------------ */
typedef struct gofft_uneven gofft_uneven;
/* count signals; signal i has lengths[i] elements at in_offsets[i] of the
 * packed input and out_offsets[i] of the packed output (elements of the
 * precision's complex type; NULL offsets = packed back to back, out = in). */
GOFFT_API int gofft_uneven_create(int precision, const int64_t *lengths, int64_t count,
                                  const int64_t *in_offsets, const int64_t *out_offsets,
                                  gofft_uneven **out);
GOFFT_API int gofft_uneven_destroy(gofft_uneven *u);
/* Forward or normalised inverse of every signal: one persistent kernel (plus a
 * counter reset) on `stream`, or in the per-phase mode one launch per phase
 * with the length classes spread over streams forked from and joined back
 * into `stream`; capturable in a CUDA graph once the batch has run on the
 * same buffers.  Errors of the device-side waits are reported by
 * gofft_uneven_status. */
GOFFT_API int gofft_uneven_exec(gofft_uneven *u, const void *in, void *out, int inverse,
                                gofft_stream stream);
/* Synchronises and returns GOFFT_ETIMEOUT if a bounded wait of the last run
 * expired (its results are then invalid). */
GOFFT_API int gofft_uneven_status(gofft_uneven *u);
/* what = 0: persistent (1, default unless the autotuner chose otherwise) or
 * one launch per phase (0);
 * 1: poll limit of the device-side waits; 2: test hook that makes one wait
 * depend on work that never completes (to exercise the timeout path). */
GOFFT_API int gofft_uneven_set(gofft_uneven *u, int what, int64_t value);
GOFFT_API int64_t gofft_uneven_describe(const gofft_uneven *u, char *buf, int64_t cap);

/* ------------------------------------------------------------------------ */
/* 2c. CUDA graphs: capture any sequence of gofft_exec_* / gofft_uneven_exec */
/*     calls on a stream and replay it.                                      */
/* ------------------------------------------------------------------------ */
typedef struct gofft_graph gofft_graph;
GOFFT_API int gofft_graph_begin(gofft_stream stream);
GOFFT_API int gofft_graph_end(gofft_stream stream, gofft_graph **out);
GOFFT_API int gofft_graph_launch(gofft_graph *g, gofft_stream stream);
GOFFT_API int gofft_graph_destroy(gofft_graph *g);

/* ------------------------------------------------------------------------ */
/* 2d. Adjoints (vector-Jacobian products) and the fused 2-D spectral filter */
/*     -- no counterpart in the reference, which has no differentiation.     */
/*     Gradients use the real inner product Re sum conj(a) b: a complex      */
/*     gradient holds dL/dRe + i dL/dIm (torch.autograd's convention for a   */
/*     real loss).  Buffers have the layouts of the plan's own transforms.   */
/* ------------------------------------------------------------------------ */

/* Adjoint of gofft_exec_c2c(p, ., ., inverse): for the forward it is the
 * unnormalised inverse (N IFFT), for the inverse the forward scaled by 1/N
 * (N = product of the plan's shape).  g and out: the plan's complex layout. */
GOFFT_API int gofft_vjp_c2c(gofft_plan *p, const void *g, void *out, int inverse, gofft_stream stream);
/* Adjoint of gofft_exec_r2c: bins g -> reals out, N IRFFT(g / w) with the
 * real-spectrum edge-bin weights w_k = 1 for k = 0 and k = n/2 (n even) along
 * the last axis, 2 otherwise.  Imaginary parts of those edge bins do not
 * contribute (the forward's outputs there are real for rank 1). */
GOFFT_API int gofft_vjp_r2c(gofft_plan *p, const void *g, void *out, gofft_stream stream);
/* Adjoint of gofft_exec_c2r (with all n/2+1 bins read): reals g -> bins out,
 * (w / N) RFFT(g).  For a short spectrum (nbins < n/2+1) the missing bins'
 * entries of out are the gradient a caller drops. */
GOFFT_API int gofft_vjp_c2r(gofft_plan *p, const void *g, void *out, gofft_stream stream);

/* 2-D spectral filter over a rank-2 real plan (batch B of R x C images):
 *   y_b = IRFFT2(H * RFFT2(x_b)),  H: R x (C/2+1) complex (shared by images).
 * Three passes per L2 block of images: row R2C, one fused column pass (column
 * FFT, multiply by H, column IFFT), row C2R.  saved (nullable): B spectra
 * RFFT2(x_b) written for the backward's dH. */
GOFFT_API int gofft_filter2_forward(gofft_plan *p, const void *x, const void *H, void *y, void *saved,
                                    gofft_stream stream);
/* Backward of gofft_filter2_forward for an upstream gradient g = dL/dy:
 *   dx   = IRFFT2(conj(H) * RFFT2(g))                      (dx nullable)
 *   dH   = sum_b conj(X_b) * (w / (R C)) * RFFT2(g_b)      (dH nullable)
 * with w the edge-bin weights of the C axis.  dH needs the forward's saved
 * spectra and a scratch buffer of the same size (B R (C/2+1) complex) for the
 * per-image terms, summed in a fixed order (reproducible); scratch may be
 * saved itself, which is then overwritten. */
GOFFT_API int gofft_vjp_filter2(gofft_plan *p, const void *g, const void *H, const void *saved, void *scratch,
                                void *dx, void *dH, gofft_stream stream);

/* ------------------------------------------------------------------------ */
/* 3. Instrumentation and tuning (no counterpart in the reference).          */
/* ------------------------------------------------------------------------ */

/* Number of engine kernels launched by this process so far. */
GOFFT_API int64_t gofft_launch_count(void);
/* Turn CUDA-event timing of every line-kernel launch on (1) or off (0): an
 * event pair is recorded on the launch stream around each launch. */
GOFFT_API int gofft_timing_enable(int on);
/* Collects the timed launches since the last report (synchronising on their
 * events) as JSON [{kernel, launches, ms, bytes}], bytes being the
 * compulsory input+output bytes.  Call once with buf == NULL to aggregate and
 * get the length, then again with a buffer to copy it. */
GOFFT_API int64_t gofft_timing_report(char *buf, int64_t cap);
/* Overrides the lines-per-CTA of the line kernel for (precision, length n,
 * op, column mode); lpc <= 0 restores the heuristic.  Used by the autotuner. */
GOFFT_API int gofft_set_lines_per_cta(int precision, int64_t n, int op, int colmode, int lpc);
/* Bytes of complex intermediate one L2 block may hold in plans created
 * afterwards: rank-2 real plans run their row and column passes per block of
 * images, complex N-D plans their last two axes per block of planes, so the
 * intermediate stays in L2.  bytes <= 0 restores the default (48 MiB).  A
 * tuning knob (process-wide); results do not depend on it. */
GOFFT_API int gofft_set_l2_block_bytes(int64_t bytes);
/* Streams ("lanes") that plans created afterwards rotate their L2 blocks
 * over: 2 (the default, 0 restores it) overlaps one block's passes with the
 * next block's; 1 runs the blocks one after another on the caller's stream
 * (each pass then runs alone, e.g. to time it).  GOFFT_EINVAL otherwise. */
GOFFT_API int gofft_set_lanes(int lanes);
/* Turns the TMA-fed persistent line kernel on (1) or off (0, the default)
 * for launches made afterwards.  When on, plain complex lines and the packed
 * real lines of even-length real transforms run on it wherever an instance
 * was built for the line's schedule: tiles are copied into a ring of
 * shared-memory slots (tensor copies for image columns, bulk copies for rows)
 * while the CTA's warp groups transform earlier tiles.  Results agree with
 * the default kernels to rounding (a tuning and comparison switch). */
GOFFT_API int gofft_set_tma_pipeline(int on);
/* Reads and clears the current device's timeout word of the pipelined line
 * kernel (synchronises the device): GOFFT_OK, or GOFFT_ETIMEOUT if one of its
 * bounded waits gave up since the last call (results of that launch are
 * then invalid).  No such wait gives up in normal operation. */
GOFFT_API int gofft_pipeline_status(void);
/* Programmatic dependent launch of the line kernels made afterwards: 0 off
 * (each kernel starts when the stream's previous one has completed), 1 each
 * line kernel may be scheduled before its predecessor in the stream has
 * finished and waits on the device until it has (its writes visible), 2 as
 * 1 with every line kernel also letting the next one be scheduled from the
 * start of its CTAs.  Results are identical in every mode.  GOFFT_EINVAL for
 * another mode. */
GOFFT_API int gofft_set_dependent_launch(int mode);
/* Selects (on = 1) the persistent double-buffered line kernel for
 * (precision, n, op) where one exists.  Used by the autotuner. */
GOFFT_API int gofft_set_pipelined(int precision, int64_t n, int op, int on);
/* Radix-schedule variant of length n in a precision, for plans created
 * afterwards (plans already created keep theirs): 0 = radices up to 16 with
 * 16 elements per thread (FP32: up to 32), the default; 1 = radices up to 8
 * with 8 elements per thread (twice the threads per line, half the
 * registers, one more stage); 2 (FP32 forms only; FP64 keeps 0) = radices up
 * to 32 with 32 elements per thread (fewer stages); uneven batches build
 * at most variant 1.  The autotuner's schedule choice. */
GOFFT_API int gofft_set_schedule(int precision, int64_t n, int variant);
GOFFT_API int gofft_get_schedule(int precision, int64_t n);

/* Autotuner (no counterpart in the reference, whose plans are fixed by
 * plan.go's router).  Times candidate settings for batch transforms of
 * `shape` on the current device -- the radix-schedule variant of each line
 * length, the lines per CTA of each pass, then the double-buffered
 * persistent kernel per pass -- keeps the fastest, and
 * leaves them set for plans created afterwards (process-wide per precision
 * and length, like FFTW wisdom).  Allocates its own buffers; takes one forward
 * and inverse transform per candidate.  Writes the resulting wisdom (JSON)
 * to `wisdom` (at most cap bytes, may be NULL) and returns its full length,
 * or minus a status on error. */
GOFFT_API int64_t gofft_autotune(int kind, int precision, const int64_t *shape, int rank, int64_t batch,
                                 char *wisdom, int64_t cap);
/* The same for an uneven batch (gofft_uneven_create's lengths): the schedule
 * variant of each length class, then the persistent launch against one
 * launch per phase (the default for uneven batches of that precision created
 * afterwards; gofft_uneven_set can still change one batch). */
GOFFT_API int64_t gofft_autotune_uneven(int precision, const int64_t *lengths, int64_t count, char *wisdom,
                                        int64_t cap);
/* Current wisdom as JSON: {"gofft_wisdom":1,"schedule":[[prec,n,variant],..],
 * "lpc":[[prec,n,op,colmode,lpc],..],"pipe":[[prec,n,op,on],..],
 * "uneven":[[prec,persistent],..]}. */
GOFFT_API int64_t gofft_wisdom_export(char *buf, int64_t cap);
/* Applies exported wisdom (entries are added to / replace the current
 * settings); GOFFT_EINVAL on a malformed document, nothing applied then. */
GOFFT_API int gofft_wisdom_import(const char *json);
/* Drops all tuning settings (defaults again for plans created afterwards). */
GOFFT_API int gofft_wisdom_forget(void);

#ifdef __cplusplus
}
#endif
#endif /* GOFFT_H */
