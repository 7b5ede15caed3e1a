// pipe.cuh -- the TMA-fed persistent line kernel.
//
// One CTA per SM walks its share of a launch's tiles (tile t, t + grid, ...).
// A tile is LPC lines: LPC adjacent columns of an image (column mode: the
// non-contiguous axis of a 2-D transform) or LPC consecutive rows (row mode).
// The tiles land in a ring of S shared-memory slots, each guarded by an
// mbarrier that completes when the slot's copies have landed.  G groups of
// warps take the tiles in turn: a group waits for its tile's slot, runs the
// compiled Stockham schedule on it in place (the first stage reads the
// unpadded copy as it landed, later stages use the bank-conflict-free padded
// layout), writes the result to global memory from the last stage, and at
// once refills the slot with the tile S places ahead.  While a group
// computes, the copies of the next tiles are already in flight, so the
// global-memory latency of a tile's first stage does not stall the SM.
//
// Copies (the fill modes):
//   PIPE_COL_TMA    column tiles by 2-D tensor copies (cp.async.bulk.tensor):
//                   boxes of LPC columns x BR rows; columns past the image's
//                   last one read as zero (out-of-bounds fill)
//   PIPE_ROW_BULK   row tiles by 1-D bulk copies (cp.async.bulk): one copy of
//                   the tile's lines when they are contiguous, else one per
//                   line; tiles whose sizes break the 16-byte rule fall back
//                   to PIPE_ROW_ASYNC
//   PIPE_COL_ASYNC, PIPE_ROW_ASYNC
//                   element copies (cp.async) by the group's threads, for
//                   layouts the bulk copies cannot address (e.g. complex64
//                   rows of 513 bins: 4104-byte pitch, not a multiple of 16);
//                   their completion arrives on the same mbarrier
//                   (cp.async.mbarrier.arrive)
//
// Every wait is bounded (spin_limit polls): past it the waiting thread sets
// *err and its group stops; before the CTA ends, one thread waits (bounded)
// for the last copy into every slot, so no copy lands in a finished CTA.
// No multicast: every copy reads this GPU's own memory into this CTA only.
#pragma once
#include <cuda.h>

#include "ops.cuh"

#define PIPE_COL_TMA 0
#define PIPE_ROW_BULK 1
#define PIPE_COL_ASYNC 2
#define PIPE_ROW_ASYNC 3

namespace gf {

struct PipeArgs {
  long long ntiles;
  int tpb;            // column mode: tiles per image
  int ncols;          // column mode: columns (lines) per image
  int lp;             // row mode: landing elements per line (n, or m+1 bins)
  int fill;           // PIPE_*
  int box_rows;       // PIPE_COL_TMA: rows per box
  long long span;     // PIPE_ROW_BULK: elements between consecutive lines (0: not uniform)
  int *err;           // set to 1 when a wait gives up
  unsigned spin_limit;
};

// ---------------------------------------------------------------------------
// mbarrier, bulk-copy and proxy-fence wrappers (PTX ISA 8.x, sm_90+).
// ---------------------------------------------------------------------------
GF_DEV uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

GF_DEV void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
GF_DEV void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
GF_DEV void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// Non-blocking test: true once the phase of parity `par` has completed.
GF_DEV bool mbar_test(uint64_t *bar, uint32_t par) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(par)
      : "memory");
  return ok != 0;
}
// Polls until the phase completes or `limit` polls have passed (backing off
// with short sleeps); false on timeout.
GF_DEV bool mbar_wait(uint64_t *bar, uint32_t par, unsigned limit) {
  for (unsigned it = 0; it < limit; it++) {
    if (mbar_test(bar, par)) return true;
    if (it >= 32) __nanosleep(it >= 1024 ? 256 : 32);
  }
  return false;
}
// Adds one pending arrival to `bar`, made once every cp.async this thread
// issued before has landed.
GF_DEV void cp_async_arrive_inc(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// 1-D bulk copy global -> shared (both 16-byte aligned, bytes a multiple of 16).
GF_DEV void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// 2-D tiled tensor copy global -> shared of the box at (x, y).
GF_DEV void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// Orders this thread's shared-memory accesses before later async-proxy
// (bulk-copy) writes to the same memory.
GF_DEV void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
GF_DEV void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// The consumer group's barrier: named barrier 1 + group over its NT threads.
template <int NT> struct GroupBar {
  static GF_DEV void sync() {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)threadIdx.x / NT), "r"(NT) : "memory");
  }
};

// Slot size (bytes, 128-aligned): the padded layout of LPC lines, which is
// never smaller than the landing copy (a line's landing pitch is at most n+1
// elements, spad_size(n) >= n+1 for n >= 16; a column box covers n rows).
template <class P, int N, int LPC> constexpr size_t pipe_slot_bytes() {
  return ((size_t)LPC * (N + N / 16 + 1) * sizeof(typename P::cpx) + 127) & ~(size_t)127;
}
// Slots, then the control words: S full barriers, G claimed items, S tags,
// the claim counter and G status words.
template <class P, int N, int LPC, int S> constexpr size_t pipe_smem_bytes() {
  return (size_t)S * pipe_slot_bytes<P, N, LPC>() + S * sizeof(uint64_t) + S * sizeof(int) + 256;
}

// ---------------------------------------------------------------------------
// Fill: copies tile t's input into `slot` and arranges for its full barrier
// (one expected arrival) to complete when everything has landed.  All NT
// threads of a consumer group call this (tid 0 issues the bulk copies; the
// element copies are spread over the group).  UE is the size of the input
// side's element unit (reals for the real forward, complex otherwise); the
// landing copy is complex element i of line l at slot[l * lp + i] (row mode)
// or slot[i * LPC + l] (column mode).
// ---------------------------------------------------------------------------
template <class P, int N, int LPC, bool COL, int UE, int NT, class BAR>
GF_DEV void pipe_fill(const KArgs &a, const PipeArgs &pa, const CUtensorMap *map, long long t,
                      typename P::cpx *slot, uint64_t *full, int tid) {
  using C = typename P::cpx;
  constexpr int E = sizeof(C);
  const char *src = (const char *)a.in.ptr;
  if constexpr (COL) {
    const long long b = t / pa.tpb;
    const int c0 = (int)(t - b * pa.tpb) * LPC;
    if (pa.fill == PIPE_COL_TMA) {
      if (tid == 0) {
        mbar_arrive_expect_tx(full, (uint32_t)(N * LPC * E));
        const int y0 = (int)(b * N);
        for (int r0 = 0; r0 < N; r0 += pa.box_rows)
          tma_load_2d(slot + (size_t)r0 * LPC, map, 2 * c0, y0 + r0, full);
      }
      return;
    }
    // element copies, one row of the tile per thread at a time; columns past
    // the image's last one copy column c0 (finite data whose results are
    // never stored)
    const long long base = b * (long long)pa.ncols;
    long long co[LPC];
#pragma unroll
    for (int l = 0; l < LPC; l++) co[l] = line_off(a.in, (uint32_t)(base + (c0 + l < pa.ncols ? c0 + l : c0)));
    const long long st = a.in.stride;
    for (int r = tid; r < N; r += NT) {
      const long long ro = (long long)r * st;
#pragma unroll
      for (int l = 0; l < LPC; l++) cp_async_n<E>(slot + r * LPC + l, src + (co[l] + ro) * UE);
    }
  } else {
    const long long line0 = t * LPC;
    const int nv = (int)((a.nlines - line0) < LPC ? (a.nlines - line0) : LPC);
    const int lp = pa.lp;
    const uint32_t line_b = (uint32_t)lp * E;
    if (pa.fill == PIPE_ROW_BULK) {
      const bool one = pa.span * UE == (long long)line_b;  // contiguous lines: one copy
      const uint32_t bytes = (uint32_t)nv * line_b;
      const char *s0 = src + line_off(a.in, (uint32_t)line0) * UE;
      // every bulk copy starts on a 16-byte boundary and moves a multiple of
      // 16 bytes (the same decision in every thread)
      bool ok = one ? (bytes % 16 == 0 && ((uintptr_t)s0 % 16) == 0) : (line_b % 16 == 0);
      if (ok && !one)
        for (int l = 0; l < nv; l++)
          ok = ok && ((uintptr_t)(src + line_off(a.in, (uint32_t)(line0 + l)) * UE) % 16) == 0;
      if (ok) {
        if (tid == 0) {
          mbar_arrive_expect_tx(full, bytes);
          if (one) {
            bulk_load(slot, s0, bytes, full);
          } else {
            for (int l = 0; l < nv; l++)
              bulk_load(slot + (size_t)l * lp, src + line_off(a.in, (uint32_t)(line0 + l)) * UE, line_b, full);
          }
        }
        return;
      }
    }
    for (int e = tid; e < nv * lp; e += NT) {
      const int l = e / lp, i = e - l * lp;
      cp_async_n<E>(slot + e, src + line_off(a.in, (uint32_t)(line0 + l)) * UE + (size_t)i * E);
    }
  }
  // element copies: each thread's copies hold the phase open until they land
  // (cp.async.mbarrier.arrive adds one pending arrival and makes it when the
  // copies complete); tid 0 then makes the expected arrival once every thread
  // has registered
  cp_async_arrive_inc(full);
  BAR::sync();
  if (tid == 0) mbar_arrive(full);
}

// ---------------------------------------------------------------------------
// Consumers: the even-length real inverse's reverse untangle (realplan.go:
// 235-272, as OpC2RPacked::prep_row) from the landed bins (m+1 per line at
// lb) into the padded packed spectrum at s; register-staged, since the
// padded line overlaps the landed ones.
// ---------------------------------------------------------------------------
template <class P, int M, int T, class BAR>
GF_DEV void c2r_prep_landed(const KArgs &a, const LineCtx &c, const Cx<P> *lb, Cx<P> *s) {
  using C = Cx<P>;
  using Rl = typename P::real;
  using TW = typename P::tw_t;
  constexpr int H = M / 2 + 1;
  constexpr int IT = (H + T - 1) / T;
  C xk[IT], xm[IT];
#pragma unroll
  for (int it = 0; it < IT; it++) {
    const int k = c.t + it * T;
    if (IT * T > H && k >= H) break;
    xk[it] = lb[k];
    xm[it] = lb[M - k];
  }
  BAR::sync();
  const TW *tw = (const TW *)a.aux0;
  const Rl half = (Rl)0.5;
  const bool wgt = (a.ic & GF_EDGE_WEIGHT) != 0;
#pragma unroll
  for (int it = 0; it < IT; it++) {
    const int k = c.t + it * T;
    if (IT * T > H && k >= H) break;
    if (k == 0) {
      const Rl x0 = xk[it].x, xmv = xm[it].x;
      s[0] = mkc((x0 + xmv) * half, -(x0 - xmv) * half);
      continue;
    }
    C v = xk[it], w = xm[it];
    if (wgt) {
      v = mkc(v.x * half, v.y * half);
      w = mkc(w.x * half, w.y * half);
    }
    const C xe = mkc((v.x + w.x) * half, (v.y - w.y) * half);
    const C d = mkc((v.x - w.x) * half, (v.y + w.y) * half);
    C xo;
    if constexpr (short_tw<P, M>()) xo = cmul(d, cconj_tw(ld_keep(&((const float2 *)a.aux1)[k])));
    else xo = twmul(d, cconj_tw(ld_keep(&tw[k])));
    s[spad(k)] = cconj(mkc(xe.x - xo.y, xe.y + xo.x));
    if (M - k != k) s[spad(M - k)] = cconj(mkc(xe.x + xo.y, -(xe.y - xo.x)));
  }
  BAR::sync();
}

// One tile of the op on the slot (all NT threads of the group).
template <class P, class Op, int N, int T, int LPC, bool COL, class S, class BAR>
GF_DEV void pipe_tile(const KArgs &a, const PipeArgs &pa, typename P::cpx *slot, long long t, int tid) {
  using C = typename P::cpx;
  LineCtx c;
  if constexpr (COL) {
    c.l = tid % LPC;
    c.t = tid / LPC;
    const long long b = t / pa.tpb;
    const int col = (int)(t - b * pa.tpb) * LPC + c.l;
    c.line = b * pa.ncols + col;
    c.valid = col < pa.ncols;
  } else {
    c.l = tid / T;
    c.t = tid % T;
    c.line = t * LPC + c.l;
    c.valid = c.line < a.nlines;
  }
  c.ioff = 0;
  c.ooff = c.valid ? line_off(a.out, (uint32_t)c.line) : 0;
  constexpr int STEP = COL ? LPC : 1;
  C *sb = COL ? slot + c.l : slot + (size_t)c.l * spad_size(N);
  const C *lb = COL ? slot + c.l : slot + (size_t)c.l * pa.lp;
  if constexpr (std::is_same<Op, OpC2RPacked>::value) {
    c2r_prep_landed<P, N, T, BAR>(a, c, lb, sb);
    run_stages_ct<P, Op, N, T, false, true, STEP, false, BAR, false>(S{}, sb, a, c, false, false, true);
  } else if constexpr (std::is_same<Op, OpR2CPacked>::value) {
    run_stages_ct<P, Op, N, T, false, false, STEP, false, BAR, true>(S{}, sb, a, c, false, false, false, lb);
    Op::template store_row<P, N, T>(a, c, sb);
  } else {
    run_stages_ct<P, Op, N, T, false, true, STEP, false, BAR, true>(S{}, sb, a, c, Op::first_conj(a), false, true,
                                                                    lb);
  }
}

// ---------------------------------------------------------------------------
// The kernel: G groups of LPC*T threads, every warp a worker (no producer
// warp: a 17th warp would cap every thread at 96 registers).  The CTA's
// tiles are blockIdx.x + i * gridDim.x, i = 0 .. mine-1; local tile i lives
// in slot i % S.  The first S tiles are copied at the start; after that the
// group that releases slot s (tile i) immediately refills it with tile i + S
// and records i + S in the slot's tag.  A group claims the next local tile
// from a counter in shared memory, waits until the slot's tag reads i (so the
// slot's previous fill has completed and the parity wait on its full barrier
// is unambiguous), then waits on the full barrier.  Claims are in order and
// every claimed tile is worked on, so each wait ends.
// ---------------------------------------------------------------------------
template <class P, class Op, int N, int T, int LPC, int G, int S, bool COL, class Sch>
__global__ void __launch_bounds__(G *LPC *T, 1)
    k_pipe(const KArgs a, const PipeArgs pa, const __grid_constant__ CUtensorMap map) {
  using C = typename P::cpx;
  using BAR = GroupBar<LPC * T>;
  constexpr int NT = LPC * T;
  constexpr int UE = std::is_same<Op, OpR2CPacked>::value ? (int)sizeof(typename P::real) : (int)sizeof(C);
  constexpr size_t SLOT = pipe_slot_bytes<P, N, LPC>();
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + S * SLOT);
  long long *s_item = reinterpret_cast<long long *>(full + S);
  volatile int *tag = reinterpret_cast<volatile int *>(s_item + G);
  int *claim = const_cast<int *>(tag + S);
  int *s_ok = claim + 1;
  auto slot = [&](int s) { return reinterpret_cast<C *>(smem + (size_t)s * SLOT); };
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      tag[s] = -1;
    }
    *claim = 0;
    fence_mbar_init();
  }
  __syncthreads();
  const long long mine = pa.ntiles > blockIdx.x ? (pa.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  const int g = threadIdx.x / NT;
  const int tid = threadIdx.x - g * NT;
  // the first S tiles
  for (long long i = g; i < S && i < mine; i += G) {
    if (tid == 0) tag[i] = (int)i;
    pipe_fill<P, N, LPC, COL, UE, NT, BAR>(a, pa, &map, blockIdx.x + i * gridDim.x, slot((int)i), &full[i], tid);
  }
  for (;;) {
    if (tid == 0) {
      const long long i = atomicAdd(claim, 1);
      int ok = 1;
      if (i < mine) {
        const int s = (int)(i % S);
        unsigned polls = 0;
        while (tag[s] != (int)i) {
          if (++polls > pa.spin_limit) {
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
        __threadfence_block();
        if (ok) ok = mbar_wait(&full[s], (uint32_t)((i / S) & 1), pa.spin_limit);
        if (!ok) atomicExch(pa.err, 1);
      }
      s_item[g] = i;
      s_ok[g] = ok;
    }
    BAR::sync();
    const long long i = s_item[g];
    if (i >= mine || !s_ok[g]) break;
    const int s = (int)(i % S);
    // each thread observes the completed phase itself (immediate: the slot
    // is refilled only by this group, after this tile)
    if (!mbar_wait(&full[s], (uint32_t)((i / S) & 1), pa.spin_limit)) atomicExch(pa.err, 1);
    pipe_tile<P, Op, N, T, LPC, COL, Sch, BAR>(a, pa, slot(s), blockIdx.x + i * gridDim.x, tid);
    // the group's shared-memory accesses to the slot come before the refill's
    // copies into it
    fence_async_smem();
    BAR::sync();
    if (i + S < mine) {
      if (tid == 0) tag[s] = (int)(i + S);
      pipe_fill<P, N, LPC, COL, UE, NT, BAR>(a, pa, &map, blockIdx.x + (i + S) * gridDim.x, slot(s), &full[s],
                                             tid);
    }
  }
  // no copy may still be landing when the CTA ends: every slot's last fill
  // has completed (bounded wait; immediate unless a group gave up)
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      const int last = tag[s];
      if (last >= 0 && !mbar_wait(&full[s], (uint32_t)((last / S) & 1), pa.spin_limit)) atomicExch(pa.err, 1);
    }
  }
}

}  // namespace gf
