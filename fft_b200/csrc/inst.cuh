// inst.cuh -- instantiates every kernel of one precision (included by the
// per-precision translation units so the three compile in parallel).
#pragma once
#include "dispatch.h"
#include "kernels.cuh"

namespace gf {

// GROUP 0: complex and convolution ops; GROUP 1: real ops.
template <class P, int M, int GROUP> KFn pick_line(int op) {
  if constexpr (GROUP == 0) {
    switch (op) {
      case OP_C2C: return k_line<P, M, OpC2C>;
      case OP_C2C_TW: return k_line<P, M, OpC2CTwiddle>;
      case OP_RADER: return k_line<P, M, OpRader>;
      case OP_BLUE: return k_line<P, M, OpBluestein>;
      case OP_RADER_FS1: return k_line<P, M, OpRaderFS1>;
      case OP_RADER_FS2: return k_line<P, M, OpRaderFS2>;
      case OP_RADER_FS4: return k_line<P, M, OpRaderFS4>;
      case OP_FILTER_COL: return k_line<P, M, OpFilterCol>;
      default: return nullptr;
    }
  } else {
    switch (op) {
      case OP_R2C: return k_line<P, M, OpR2CPacked>;
      case OP_C2R: return k_line<P, M, OpC2RPacked>;
      case OP_R2C_FULL: return k_line<P, M, OpR2CFull>;
      case OP_C2R_FULL: return k_line<P, M, OpC2RFull>;
      case OP_SPECTRO: return k_line<P, M, OpSpectro>;
      default: return nullptr;
    }
  }
}

// FP64 lines use 16 register elements per thread (32 would spill); the FP32
// forms also get a 32-element variant for lines longer than 16 x 512.
template <class P, int GROUP> KFn pick_maxe(int maxe, int op) {
  // 8-element schedules run in the 16-element kernel (the second register
  // half stays unused)
  if (maxe <= 16) return pick_line<P, 16, GROUP>(op);
  if constexpr (sizeof(typename P::cpx) == 8) {
    if (maxe == 32) return pick_line<P, 32, GROUP>(op);
  }
  return nullptr;
}

// Compile-time schedules: (N, threads per line, lines per CTA, row-ops too,
// radices...).  Each length has the run-time heuristic's lines per CTA and
// twice that (column transforms of FP32 data); the schedules are those
// gpu_radices() and pick_threads() derive for the length, the default
// variant first, then the radix-8 variant (8 elements per thread) and the
// FP32 radix-32 variant (32 elements per thread) for the lengths of the 2-D
// workloads, then fewer lines per CTA for small complex batches.
#define GF_CT_LIST(X)                                                     \
  X(64, 4, 64, 1, 8, 8) X(64, 4, 128, 0, 8, 8)                           \
  X(128, 8, 32, 1, 16, 8) X(128, 8, 64, 0, 16, 8)                        \
  X(256, 16, 16, 1, 16, 16) X(256, 16, 32, 0, 16, 16)                    \
  X(512, 32, 8, 1, 8, 8, 8) X(512, 32, 16, 0, 8, 8, 8)                   \
  X(1024, 64, 4, 1, 16, 8, 8) X(1024, 64, 8, 0, 16, 8, 8)                \
  X(2048, 128, 2, 1, 16, 16, 8) X(2048, 128, 4, 0, 16, 16, 8)            \
  X(4096, 256, 1, 1, 16, 16, 16) X(4096, 256, 2, 0, 16, 16, 16)          \
  X(8192, 512, 1, 1, 16, 8, 8, 8)                                         \
  X(16384, 512, 1, 1, 16, 16, 8, 8)                                       \
  X(256, 32, 8, 1, 8, 8, 4) X(256, 32, 16, 0, 8, 8, 4)                   \
  X(512, 64, 4, 1, 8, 8, 8) X(512, 64, 8, 0, 8, 8, 8)                    \
  X(1024, 128, 2, 1, 8, 8, 4, 4) X(1024, 128, 4, 0, 8, 8, 4, 4)          \
  X(2048, 256, 1, 1, 8, 8, 8, 4) X(2048, 256, 2, 0, 8, 8, 8, 4)          \
  X(512, 16, 16, 1, 32, 16) X(1024, 32, 8, 1, 32, 32)                     \
  X(128, 8, 2, 0, 16, 8) X(256, 16, 2, 0, 16, 16) X(256, 16, 4, 0, 16, 16) \
  X(512, 32, 2, 0, 8, 8, 8)                                               \
  X(1024, 64, 1, 0, 16, 8, 8) X(1024, 64, 2, 0, 16, 8, 8)                 \
  X(512, 64, 2, 1, 8, 8, 8) X(512, 32, 4, 1, 8, 8, 8) X(256, 16, 8, 1, 16, 16)

template <int... Rs> constexpr bool sched_eq(const int *r, int nst) {
  constexpr int a[] = {Rs...};
  if (nst != (int)sizeof...(Rs)) return false;
  for (int i = 0; i < nst; i++)
    if (a[i] != r[i]) return false;
  return true;
}

#ifndef GF_F32_MINB
#define GF_F32_MINB 3
#endif

// GROUP 0: complex ops (C2C, four-step twiddle); GROUP 1: real-row ops.
// PIPE selects the persistent double-buffered kernel.
template <class P, int GROUP, int N, int T, int L, bool ROWOPS, int... Rs> KFn ct_for(int op, bool pipe) {
  using S = Sched<Rs...>;
  // FP64 radix-16 butterflies need ~128 registers (two 256-thread CTAs per
  // SM); the FP32 forms and the 8-element schedules fit in fewer, so ask for
  // more resident CTAs (more warps to hide shared-memory and twiddle
  // latency): 8-element schedules get 64 registers a thread, 32-element
  // (FP32) ones 128.
  constexpr int E = ct_maxe_r<N, T, Rs...>();
  constexpr int MINB = (E <= 8)    ? (65536 / (L * T * 64) > 0 ? 65536 / (L * T * 64) : 1)
                       : (E >= 32) ? (65536 / (L * T * 128) > 0 ? 65536 / (L * T * 128) : 1)
                       : (L * T <= 256) ? (sizeof(typename P::cpx) == 16 ? 2 : GF_F32_MINB) : 1;
  if constexpr (sizeof(typename P::cpx) == 16 && E > 16) {
    return nullptr;  // 32-element FP64 schedules would spill; not built
  } else if constexpr (N == 16384 && sizeof(typename P::cpx) == 16) {
    return nullptr;  // FP64 16384 is two-pass
  } else if constexpr (GROUP == 0) {
    switch (op) {
      case OP_C2C: return pipe ? k_line_pp<P, N, T, L, MINB, OpC2C, S> : k_line_ct<P, N, T, L, MINB, OpC2C, S>;
      case OP_C2C_TW:
        return pipe ? k_line_pp<P, N, T, L, MINB, OpC2CTwiddle, S> : k_line_ct<P, N, T, L, MINB, OpC2CTwiddle, S>;
      case OP_FILTER_COL: return pipe ? nullptr : k_line_ct<P, N, T, L, MINB, OpFilterCol, S>;
      default: return nullptr;
    }
  } else if constexpr (ROWOPS) {
    switch (op) {
      case OP_R2C:
        return pipe ? k_line_pp<P, N, T, L, MINB, OpR2CPacked, S> : k_line_ct<P, N, T, L, MINB, OpR2CPacked, S>;
      case OP_C2R:
        return pipe ? k_line_pp<P, N, T, L, MINB, OpC2RPacked, S> : k_line_ct<P, N, T, L, MINB, OpC2RPacked, S>;
      case OP_SPECTRO: return pipe ? nullptr : k_line_ct<P, N, T, L, MINB, OpSpectro, S>;
      default: return nullptr;
    }
  } else {
    return nullptr;
  }
}

template <class P, int GROUP> KFn pick_ct(int n, int T, int lpc, int op, const int *rad, int nst, bool pipe) {
#define GF_CT_X(N, TT, L, ROW, ...)                                           \
  if (n == N && T == TT && lpc == L && sched_eq<__VA_ARGS__>(rad, nst))      \
    return ct_for<P, GROUP, N, TT, L, ROW != 0, __VA_ARGS__>(op, pipe);
  GF_CT_LIST(GF_CT_X)
#undef GF_CT_X
  return nullptr;
}

// Compiled schedules the persistent (uneven-batch) kernel runs: the default
// schedule of every power-of-two length up to 4096 at its row- and
// column-layout lines per CTA.
#define GF_PERSIST_LIST(X)                                                               \
  X(64, 4, 64, 8, 8) X(64, 4, 128, 8, 8) X(128, 8, 32, 16, 8) X(128, 8, 64, 16, 8)     \
  X(256, 16, 16, 16, 16) X(256, 16, 32, 16, 16) X(512, 32, 8, 8, 8, 8)                \
  X(512, 32, 16, 8, 8, 8) X(1024, 64, 4, 16, 8, 8) X(1024, 64, 8, 16, 8, 8)           \
  X(2048, 128, 2, 16, 16, 8) X(2048, 128, 4, 16, 16, 8) X(4096, 256, 1, 16, 16, 16)   \
  X(4096, 256, 2, 16, 16, 16)

template <class P> GF_DEV bool persist_ct(const KArgs &a, int op, long long tile, bool active) {
  const int n = a.lp.n, T = a.lp.T, L = a.lpc;
#define GF_PX(N, TT, LL, ...)                                                                   \
  if (n == N && T == TT && L == LL && sched_eq<__VA_ARGS__>(a.lp.radix, a.lp.nst)) {           \
    if (op == OP_C2C) persist_ct_body<P, N, TT, LL, OpC2C, Sched<__VA_ARGS__>>(a, tile, active); \
    else persist_ct_body<P, N, TT, LL, OpC2CTwiddle, Sched<__VA_ARGS__>>(a, tile, active);      \
    return true;                                                                               \
  }
  GF_PERSIST_LIST(GF_PX)
#undef GF_PX
  return false;
}

static inline int ew_blocks(long long total) {
  long long b = (total + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace gf

#define GF_DEFINE_PREC(P, SUFFIX)                                                              \
  namespace gf {                                                                               \
  const void *persist_kernel_##SUFFIX() { return (const void *)k_persist<P>; }                \
  namespace prec_##SUFFIX {                                                                    \
  using C = P::cpx;                                                                            \
  using SP = P::sp_t;                                                                          \
  using TW = P::tw_t;                                                                          \
  cudaError_t gather(void *dst, const Side &src, const EwArgs &e, cudaStream_t st) {           \
    k_gather<C><<<ew_blocks(e.nlines * e.ldst), 256, 0, st>>>(                                \
        (C *)dst, src, e.nlines, e.len, e.ldst, e.perm,                                        \
        (const std::conditional<sizeof(C) == 16, double2, float4>::type *)e.chirp, e.cj,       \
        (C *)e.x0s);                                                                           \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t spec_mul(void *y, const void *B, const EwArgs &e, cudaStream_t st) {             \
    k_spec_mul<C, SP><<<ew_blocks(e.nlines * e.len), 256, 0, st>>>(                           \
        (C *)y, (const SP *)B, e.nlines, e.len, (const C *)e.x0s, (C *)e.dc);                  \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t rader_scatter(const Side &dst, const void *y, const int *iperm, const EwArgs &e, \
                            cudaStream_t st) {                                                 \
    k_rader_scatter<C><<<ew_blocks(e.nlines * e.p), 256, 0, st>>>(                            \
        dst, (const C *)y, e.nlines, e.p, e.len, e.off, iperm, (const C *)e.x0s,               \
        (const C *)e.dc, e.cj, e.scale);                                                       \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t blue_unchirp(const Side &dst, const void *y, const EwArgs &e, cudaStream_t st) { \
    k_blue_unchirp<C, SP><<<ew_blocks(e.nlines * e.p), 256, 0, st>>>(                         \
        dst, (const C *)y, e.nlines, e.p, e.len, (const SP *)e.chirp, e.cj, e.scale);          \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t scatter(const Side &dst, const void *src, const EwArgs &e, cudaStream_t st) {    \
    k_scatter<C><<<ew_blocks(e.nlines * e.len), 256, 0, st>>>(dst, (const C *)src, e.nlines,  \
                                                              e.len, e.cj, e.scale);           \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t stage_tw(void *tw, const StageTab &t, long long total, cudaStream_t st) {        \
    k_gen_stage_tw<TW><<<ew_blocks(total), 256, 0, st>>>((TW *)tw, t, total);                 \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t roots(void *tw, long long L, long long count, cudaStream_t st) {                 \
    k_gen_roots<TW><<<ew_blocks(count), 256, 0, st>>>((TW *)tw, L, count, 1);                 \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t roots_step(void *tw, long long L, long long count, long long step, cudaStream_t st) { \
    k_gen_roots<TW><<<ew_blocks(count), 256, 0, st>>>((TW *)tw, L, count, step);              \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t spectrum(void *dst, const double2 *src, double s, long long n, cudaStream_t st) { \
    k_store_spectrum<SP><<<ew_blocks(n), 256, 0, st>>>((SP *)dst, src, s, n);                 \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t untangle(const Side &dst, const void *Z, long long nl, int m, const void *tw,    \
                       double wsc, cudaStream_t st) {                                          \
    k_untangle<C, TW><<<ew_blocks(nl * (m / 2 + 1)), 256, 0, st>>>(dst, (const C *)Z, nl, m, \
                                                                   (const TW *)tw, wsc);       \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t reverse_untangle(void *Z, const Side &src, long long nl, int m, int nb,          \
                               const void *tw, int halve, cudaStream_t st) {                   \
    k_reverse_untangle<C, TW><<<ew_blocks(nl * (m / 2 + 1)), 256, 0, st>>>(                   \
        (C *)Z, src, nl, m, nb, (const TW *)tw, halve);                                        \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t promote(void *dst, const Side &src, long long nl, int n, cudaStream_t st) {      \
    k_promote<C><<<ew_blocks(nl * n), 256, 0, st>>>((C *)dst, src, nl, n);                    \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t copy_bins(const Side &dst, const void *src, long long nl, int n, double wsc,     \
                        cudaStream_t st) {                                                     \
    k_copy_bins<C><<<ew_blocks(nl * (n / 2 + 1)), 256, 0, st>>>(dst, (const C *)src, nl, n,   \
                                                                wsc);                          \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t mirror(void *dst, const Side &src, long long nl, int n, int nb, int halve,       \
                     cudaStream_t st) {                                                        \
    k_mirror<C><<<ew_blocks(nl * n), 256, 0, st>>>((C *)dst, src, nl, n, nb, halve);          \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t take_real(const Side &dst, const void *src, long long nl, int n, double scale,   \
                        cudaStream_t st) {                                                     \
    k_take_real<C><<<ew_blocks(nl * n), 256, 0, st>>>(dst, (const C *)src, nl, n, scale);     \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t sum_batches(void *dst, const void *part, long long count, long long nb,          \
                          cudaStream_t st) {                                                   \
    k_sum_batches<C><<<ew_blocks(count), 256, 0, st>>>((C *)dst, (const C *)part, count, nb); \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  cudaError_t filter_ew(void *spec, const void *H, void *saved, void *part, long long nb,      \
                        long long R, long long K, long long cols, int fl, double dsc,          \
                        cudaStream_t st) {                                                     \
    k_filter_ew<C><<<ew_blocks(nb * R * K), 256, 0, st>>>((C *)spec, (const C *)H, (C *)saved, \
                                                          (C *)part, nb, R, K, cols, fl, dsc); \
    return cudaGetLastError();                                                                 \
  }                                                                                            \
  }                                                                                            \
  }

// Compile-time-schedule instances of one precision and op group (their own
// translation units, so the build parallelises).
#define GF_DEFINE_CT(P, SUFFIX, GROUP)                                                         \
  namespace gf {                                                                               \
  KFn line_kernel_ct_##SUFFIX##_##GROUP(int n, int T, int lpc, int op, const int *rad, int nst,   \
                                        bool pipe) {                                           \
    return pick_ct<P, GROUP>(n, T, lpc, op, rad, nst, pipe);                                   \
  }                                                                                            \
  }

// Run-time-schedule instances of one precision and op group.
#define GF_DEFINE_GEN(P, SUFFIX, GROUP)                                                        \
  namespace gf {                                                                               \
  KFn line_kernel_##SUFFIX##_##GROUP(int maxe, int op) { return pick_maxe<P, GROUP>(maxe, op); } \
  }
