// dispatch.h -- host-visible handles to the per-precision kernel instances.
#pragma once
#include <cuda_runtime.h>
#include "ops.cuh"

namespace gf {

enum Prec { F64 = 0, F32 = 1, F32C = 2 };
enum Op {
  OP_C2C = 0,      // plain complex line
  OP_C2C_TW = 1,   // four-step pass 1 (twiddled epilogue)
  OP_R2C = 2,      // even real forward (packed)
  OP_C2R = 3,      // even real inverse (packed)
  OP_R2C_FULL = 4, // real forward through a full complex line
  OP_C2R_FULL = 5, // real inverse through the Hermitian mirror
  OP_RADER = 6,    // fused Rader convolution
  OP_BLUE = 7,     // fused Bluestein convolution
  OP_SPECTRO = 8,  // fused spectrogram frame
  OP_RADER_FS1 = 9,   // two-pass Rader: gathered column pass
  OP_RADER_FS2 = 10,  // two-pass Rader: row pass with spectrum multiply
  OP_RADER_FS4 = 11,  // two-pass Rader: row pass with the output scatter
  OP_FILTER_COL = 12, // 2-D spectral filter: column FFT, multiply, column IFFT
  OP_RADER_IP = 13,   // Rader with the whole convolution in shared memory (rader_ip.cuh)
  OP_COUNT = 14
};

typedef void (*KFn)(KArgs);

// Run-time-schedule line kernel for (maxe, op) in each precision and op group
// (0: complex and convolution ops, 1: real ops); nullptr if not instantiated.
KFn line_kernel_f64_0(int maxe, int op);
KFn line_kernel_f64_1(int maxe, int op);
KFn line_kernel_f32_0(int maxe, int op);
KFn line_kernel_f32_1(int maxe, int op);
KFn line_kernel_f32c_0(int maxe, int op);
KFn line_kernel_f32c_1(int maxe, int op);
// Compile-time-schedule instance for (n, threads per line, lines per CTA, op,
// schedule), or nullptr.
// (group 0: C2C and four-step twiddle; group 1: real-row ops; pipe: the
// persistent double-buffered variant)
KFn line_kernel_ct_f64_0(int n, int T, int lpc, int op, const int *rad, int nst, bool pipe);
KFn line_kernel_ct_f64_1(int n, int T, int lpc, int op, const int *rad, int nst, bool pipe);
KFn line_kernel_ct_f32_0(int n, int T, int lpc, int op, const int *rad, int nst, bool pipe);
KFn line_kernel_ct_f32_1(int n, int T, int lpc, int op, const int *rad, int nst, bool pipe);
KFn line_kernel_ct_f32c_0(int n, int T, int lpc, int op, const int *rad, int nst, bool pipe);
KFn line_kernel_ct_f32c_1(int n, int T, int lpc, int op, const int *rad, int nst, bool pipe);

// Elementwise / table kernels of one precision, launched on `st`.
struct EwArgs {
  long long nlines;
  int len, ldst, off, p;
  const int *perm;
  const void *chirp;  // sp_t table
  int cj;
  double scale;
  void *x0s, *dc;
};

#define GF_DECLARE_PREC(SUFFIX)                                                               \
  namespace prec_##SUFFIX {                                                                   \
  cudaError_t gather(void *dst, const Side &src, const EwArgs &e, cudaStream_t st);           \
  cudaError_t spec_mul(void *y, const void *B, const EwArgs &e, cudaStream_t st);             \
  cudaError_t rader_scatter(const Side &dst, const void *y, const int *iperm, const EwArgs &e, \
                            cudaStream_t st);                                                 \
  cudaError_t blue_unchirp(const Side &dst, const void *y, const EwArgs &e, cudaStream_t st); \
  cudaError_t scatter(const Side &dst, const void *src, const EwArgs &e, cudaStream_t st);    \
  cudaError_t stage_tw(void *tw, const StageTab &t, long long total, cudaStream_t st);        \
  cudaError_t roots(void *tw, long long L, long long count, cudaStream_t st);                 \
  cudaError_t roots_step(void *tw, long long L, long long count, long long step, cudaStream_t st); \
  cudaError_t spectrum(void *dst, const double2 *src, double s, long long n, cudaStream_t st); \
  cudaError_t untangle(const Side &dst, const void *Z, long long nl, int m, const void *tw,   \
                       double wsc, cudaStream_t st);                                          \
  cudaError_t reverse_untangle(void *Z, const Side &src, long long nl, int m, int nb,         \
                               const void *tw, int halve, cudaStream_t st);                   \
  cudaError_t promote(void *dst, const Side &src, long long nl, int n, cudaStream_t st);      \
  cudaError_t copy_bins(const Side &dst, const void *src, long long nl, int n, double wsc,    \
                        cudaStream_t st);                                                     \
  cudaError_t mirror(void *dst, const Side &src, long long nl, int n, int nb, int halve,      \
                     cudaStream_t st);                                                        \
  cudaError_t take_real(const Side &dst, const void *src, long long nl, int n, double scale,  \
                        cudaStream_t st);                                                     \
  cudaError_t sum_batches(void *dst, const void *part, long long count, long long nb,         \
                          cudaStream_t st);                                                   \
  cudaError_t filter_ew(void *spec, const void *H, void *saved, void *part, long long nb,     \
                        long long R, long long K, long long cols, int fl, double dsc,         \
                        cudaStream_t st);                                                     \
  }
// Plan-time integer and chirp tables (FP64 / exact integer work).
cudaError_t gen_rader_perm(int *perm, int *iperm, long long p, long long g, cudaStream_t st);
cudaError_t gen_rader_kernel(double2 *b, const int *perm, long long p, long long cl, int cyclic,
                             cudaStream_t st);
cudaError_t gen_chirp(long long *jj, double2 *w, long long n, cudaStream_t st);
cudaError_t gen_blue_kernel(double2 *b, const double2 *w, long long n, long long m, cudaStream_t st);
// The in-shared-memory Rader kernel (k_rader_ip) of each precision and its
// threads per CTA.
const void *rader_ip_kernel_f64(int *threads);
const void *rader_ip_kernel_f32(int *threads);
const void *rader_ip_kernel_f32c(int *threads);
// the two-CTA (cluster) form of the same transform
const void *rader_ip2_kernel_f64(int *threads);
const void *rader_ip2_kernel_f32(int *threads);
const void *rader_ip2_kernel_f32c(int *threads);
// The persistent multi-phase kernel (k_persist) of each precision.
const void *persist_kernel_f64();
const void *persist_kernel_f32();
const void *persist_kernel_f32c();

// Window of `kind` (0 Hann, 1 Hamming, 2 Blackman, 3 Blackman-Harris,
// 4 Bartlett), n samples of prec_bytes (8 or 4) each.
cudaError_t gen_window(void *w, int prec_bytes, long long n, int kind, cudaStream_t st);

GF_DECLARE_PREC(f64)
GF_DECLARE_PREC(f32)
GF_DECLARE_PREC(f32c)

}  // namespace gf
