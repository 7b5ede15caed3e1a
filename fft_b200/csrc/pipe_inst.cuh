// pipe_inst.cuh -- the compiled instances of the TMA-fed persistent line
// kernel (k_pipe) of one precision, and their lookup.
#pragma once
#include "dispatch.h"
#include "pipe.h"
#include "pipe.cuh"

namespace gf {

// Ops an instance is built for (bit mask).
#define PIPE_OPS_C2C 1
#define PIPE_OPS_R2C 2
#define PIPE_OPS_C2R 4

// (N, threads per line, lines per tile, consumer groups, slots, column mode,
//  ops, radices...): the schedules the plans build for the lengths of the
// 2-D real round trip (1024-point columns; 512-point packed rows of
// 1024-real images, radix-8 at 8 or 16 elements per thread) and for batched
// 1024-point complex rows.
#define GF_PIPE_LIST_F64(X)                                     \
  X(1024, 64, 4, 2, 3, 1, PIPE_OPS_C2C, 16, 8, 8)               \
  X(1024, 128, 4, 2, 3, 1, PIPE_OPS_C2C, 8, 8, 4, 4)            \
  X(1024, 64, 4, 2, 3, 0, PIPE_OPS_C2C, 16, 8, 8)               \
  X(512, 64, 4, 3, 6, 0, PIPE_OPS_R2C | PIPE_OPS_C2R, 8, 8, 8)  \
  X(512, 32, 8, 2, 3, 0, PIPE_OPS_R2C | PIPE_OPS_C2R, 8, 8, 8)

#define GF_PIPE_LIST_F32(X)                                     \
  X(1024, 64, 4, 3, 6, 1, PIPE_OPS_C2C, 16, 8, 8)               \
  X(1024, 128, 4, 2, 6, 1, PIPE_OPS_C2C, 8, 8, 4, 4)            \
  X(512, 64, 4, 4, 12, 0, PIPE_OPS_R2C | PIPE_OPS_C2R, 8, 8, 8) \
  X(512, 32, 8, 3, 6, 0, PIPE_OPS_R2C | PIPE_OPS_C2R, 8, 8, 8)

template <int... Rs> constexpr bool sched_is(const int *r, int nst) {
  constexpr int a[] = {Rs...};
  if (nst != (int)sizeof...(Rs)) return false;
  for (int i = 0; i < nst; i++)
    if (a[i] != r[i]) return false;
  return true;
}

template <class P, int N, int T, int L, int G, int S, bool COL, int OPS, int... Rs>
PipeInst pipe_for(int op) {
  using Sc = Sched<Rs...>;
  PipeInst r{};
  r.lpc = L;
  r.groups = G;
  r.slots = S;
  r.threads = G * L * T;
  r.smem = pipe_smem_bytes<P, N, L, S>();
  r.fn = nullptr;
  if constexpr ((OPS & PIPE_OPS_C2C) != 0) {
    if (op == OP_C2C) r.fn = (const void *)k_pipe<P, OpC2C, N, T, L, G, S, COL, Sc>;
  }
  if constexpr (!COL && (OPS & PIPE_OPS_R2C) != 0) {
    if (op == OP_R2C) r.fn = (const void *)k_pipe<P, OpR2CPacked, N, T, L, G, S, false, Sc>;
  }
  if constexpr (!COL && (OPS & PIPE_OPS_C2R) != 0) {
    if (op == OP_C2R) r.fn = (const void *)k_pipe<P, OpC2RPacked, N, T, L, G, S, false, Sc>;
  }
  return r;
}

template <class P, bool F64LIST>
PipeInst pipe_pick(int op, int n, int T, const int *rad, int nst, bool col) {
#define GF_PIPE_X(N, TT, L, G, S, COL, OPS, ...)                                   \
  if (n == N && T == TT && col == (COL != 0) && sched_is<__VA_ARGS__>(rad, nst)) { \
    PipeInst r = pipe_for<P, N, TT, L, G, S, COL != 0, OPS, __VA_ARGS__>(op);     \
    if (r.fn) return r;                                                            \
  }
  if constexpr (F64LIST) {
    GF_PIPE_LIST_F64(GF_PIPE_X)
  } else {
    GF_PIPE_LIST_F32(GF_PIPE_X)
  }
#undef GF_PIPE_X
  return PipeInst{};
}

}  // namespace gf

#define GF_DEFINE_PIPE(P, SUFFIX, F64LIST)                                                       \
  namespace gf {                                                                                 \
  PipeInst pipe_kernel_##SUFFIX(int op, int n, int T, const int *rad, int nst, bool col) {      \
    return pipe_pick<P, F64LIST>(op, n, T, rad, nst, col);                                      \
  }                                                                                              \
  }
