// engine.cuh -- the B200 line-FFT engine: line programs, shared-memory
// layout, the Stockham stage and the tile loops.
//
// A "line" is one 1-D transform of length n held entirely in one CTA's shared
// memory.  A CTA processes `lpc` lines of the same length at once; `T` threads
// work on each line.  The transform is a self-sorting (Stockham) mixed-radix
// decimation-in-time schedule: stage s with radix R and sub-length Ns reads
// butterfly j's inputs at j + r*(n/R), multiplies input r by
// W_{Ns*R}^{(j mod Ns)*r}, runs a straight-line DFT-R on registers and writes
// output r to (j / Ns)*Ns*R + (j mod Ns) + r*Ns.  No digit-reversal pass is
// needed; the last stage leaves natural order.
//
// Each stage is register-staged: every thread loads all of its butterflies'
// inputs, the CTA synchronises, then each thread computes and writes its
// outputs back over the same buffer (one buffer per line).  The first stage
// can read its inputs straight from global memory and the last stage can
// write straight to global memory ("direct" stages), so a transform of S
// stages makes S-1 shared-memory round trips instead of S+1.  Direct stages
// are coalesced because the thread mapping follows the layout: along a line
// (row mode) or across adjacent lines (column mode, for axes that are not
// contiguous).  Ops that need pairs of elements (real-signal packing) or a
// gather the stage cannot express use the cooperative tile loops with
// asynchronous copies instead.
#pragma once
#include <type_traits>
#include "codelets.cuh"

#define GF_MAXST 24

// KArgs::flags
#define GF_COLMAP 1        // thread mapping and smem layout across lines
#define GF_FIRST_DIRECT 2  // first stage reads global memory
#define GF_LAST_DIRECT 4   // last stage writes global memory
#define GF_PDL_TRIGGER 16  // let the stream's next (dependent) launch start its CTAs early

namespace gf {

struct LineProg {
  int n;    // line length
  int nst;  // number of stages
  int T;    // threads per line
  int maxe; // register elements per thread the schedule was sized for
  int radix[GF_MAXST];
  int ns[GF_MAXST];
  int twoff[GF_MAXST];  // offset of the stage's twiddle planes in tw
  FastDiv nsdiv[GF_MAXST];
  const void *tw;       // per-stage twiddles: plane (r-1) holds W_{Ns R}^{k r}, k < Ns
  const void *tw_hi;    // FP32-mixed programs: the same table as FP32 hi parts only
};

// FP32-mixed lines up to this length apply the hi parts of their FP64-derived
// twiddles with plain products (one FP32 rounding per twiddle keeps them well
// inside the 1e-6 relative-L2 budget); longer lines use the compensated
// hi+lo products.
#define GF_F32C_SHORT_MAX 4096
template <class P, int N> constexpr bool short_tw() {
  return std::is_same<typename P::tw_t, float4>::value && N <= GF_F32C_SHORT_MAX;
}

// Addressing of one side of a batched, strided set of lines (in elements).
// line l, element i:  base(l / lpb) + (l % lpb) * dist_l + i * stride, with
// base(b) = b * dist_b, or boff[b] when a per-batch offset table is given
// (signals of one length scattered through an uneven batch).
struct Side {
  void *ptr;
  long long dist_b, dist_l, stride;
  FastDiv lpb;
  const long long *boff;
};

GF_HD long long line_off(const Side &s, uint32_t l) {
  uint32_t b, r;
  s.lpb.divmod(l, b, r);
#ifdef __CUDA_ARCH__
  const long long base = s.boff ? __ldg(&s.boff[b]) : (long long)b * s.dist_b;
#else
  const long long base = s.boff ? s.boff[b] : (long long)b * s.dist_b;
#endif
  return base + (long long)r * s.dist_l;
}

// Stage layout used to generate the twiddle planes of a LineProg.
struct StageTab {
  int nst;
  int radix[GF_MAXST];
  int ns[GF_MAXST];
  int twoff[GF_MAXST];
};

struct KArgs {
  LineProg lp;
  Side in, out;
  long long nlines;
  int lpc;           // lines per CTA
  int flags;         // GF_COLMAP | GF_FIRST_DIRECT | GF_LAST_DIRECT
  FastDiv ndiv;      // divide by the line length n
  FastDiv lpcdiv;    // divide by lpc
  int cj_in;         // conjugate on load  (first pass of an inverse)
  int cj_out;        // conjugate on store (last pass of an inverse)
  double scale;      // applied on store
  // op-specific operands
  const void *aux0, *aux1, *aux2;
  long long ia, ib;  // integer operands (op-defined)
  int ic;
  double da;
};

// ---------------------------------------------------------------------------
// Shared-memory layout of a CTA's lines.  Row mode: line-major, each line
// padded (one spare element every 16).  Column mode: element-major with the
// lpc lines interleaved, so consecutive threads (consecutive lines) touch
// consecutive words.  A per-line view carries its base and element step.
// ---------------------------------------------------------------------------
template <class C> GF_DEV C *smem_base() {
  extern __shared__ __align__(16) unsigned char g_smem[];
  return reinterpret_cast<C *>(g_smem);
}

template <class C> struct LineView {
  C *b;
  int step;
  GF_DEV C &operator[](int i) const { return b[spad(i) * step]; }
};

// View of local line l in the tile buffer starting at sbase (the dynamic
// shared memory by default; persistent kernels alternate two buffers).
template <class C> GF_DEV LineView<C> line_view(const KArgs &a, int l, void *sbase = nullptr) {
  C *s = sbase ? reinterpret_cast<C *>(sbase) : smem_base<C>();
  LineView<C> v;
  if (a.flags & GF_COLMAP) {
    v.b = s + l;
    v.step = a.lpc;
  } else {
    v.b = s + (size_t)l * spad_size(a.lp.n);
    v.step = 1;
  }
  return v;
}

// Two spare complex slots per line after the lpc line buffers.
template <class C> GF_DEV C *line_extra(const KArgs &a, int l) {
  return smem_base<C>() + (size_t)a.lpc * spad_size(a.lp.n) + 2 * l;
}

// Per-thread context of a line kernel.
struct LineCtx {
  int l, t;              // local line, thread within the line
  long long line;        // global line index
  bool valid;            // line < nlines
  long long ioff, ooff;  // element offsets of the line on the in / out sides
};

// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async).
// ---------------------------------------------------------------------------
GF_DEV void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
GF_DEV void cp_async8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
GF_DEV void cp_async4(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
GF_DEV void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
template <int BYTES> GF_DEV void cp_async_n(void *s, const void *g) {
  if constexpr (BYTES == 16) cp_async16(s, g);
  else if constexpr (BYTES == 8) cp_async8(s, g);
  else cp_async4(s, g);
}

// ---------------------------------------------------------------------------
// Stockham stage.  FG: inputs come from Op::gload (global memory) instead of
// shared memory; TG: outputs go to Op::gstore instead of shared memory.
// ---------------------------------------------------------------------------
template <class P, class Op, int R, int MAXE, bool FG, bool TG>
GF_DEV void stage(typename P::cpx (&v)[MAXE], const LineView<typename P::cpx> &s, const KArgs &a,
                  const LineCtx &c, int ns, FastDiv nsd, const typename P::tw_t *tw, bool cj) {
  using C = typename P::cpx;
  constexpr int NB = MAXE / R;
  const int n = a.lp.n, T = a.lp.T;
  const int nb = n / R;
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int j = c.t + b * T;
    if (j < nb) {
#pragma unroll
      for (int r = 0; r < R; r++) {
        C x;
        if constexpr (FG) x = Op::template gload<P>(a, c, j + r * nb);
        else x = s[j + r * nb];
        if (cj) x.y = -x.y;
        v[b * R + r] = x;
      }
    }
  }
  if constexpr (!FG) __syncthreads();
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int j = c.t + b * T;
    if (j < nb) {
      uint32_t q, k;
      nsd.divmod((uint32_t)j, q, k);
      if (ns > 1) {
#pragma unroll
        for (int r = 1; r < R; r++)
          v[b * R + r] = twmul(v[b * R + r], ld_keep(&tw[(r - 1) * ns + k]));
      }
      Dft<R, C>::run(&v[b * R]);
      const int base = (int)q * ns * R + (int)k;
#pragma unroll
      for (int r = 0; r < R; r++) {
        if constexpr (TG) Op::template gstore<P>(a, c, base + r * ns, v[b * R + r]);
        else s[base + r * ns] = v[b * R + r];
      }
    }
  }
  if constexpr (!TG) __syncthreads();
}

template <class P, class Op, int MAXE, bool FG, bool TG>
GF_DEV void stage_sw(int R, typename P::cpx (&v)[MAXE], const LineView<typename P::cpx> &s,
                     const KArgs &a, const LineCtx &c, int ns, FastDiv nsd,
                     const typename P::tw_t *tw, bool cj) {
  switch (R) {
    case 2: stage<P, Op, 2, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 3: stage<P, Op, 3, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 4: stage<P, Op, 4, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 5: stage<P, Op, 5, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 7: stage<P, Op, 7, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 8: stage<P, Op, 8, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 11: stage<P, Op, 11, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 13: stage<P, Op, 13, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 16: stage<P, Op, 16, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj); break;
    case 32:
      if constexpr (MAXE >= 32) stage<P, Op, 32, MAXE, FG, TG>(v, s, a, c, ns, nsd, tw, cj);
      break;
    default: break;
  }
}

// Runs every stage of lp on the line view s.  All threads of the CTA call
// this (stages contain CTA barriers).  One register array serves every radix:
// giving each radix case its own array makes ptxas allocate the switch
// alternatives jointly and spill.  cj_first conjugates the first stage's
// inputs.  first_g / last_g select the direct first / last stage (the op
// must provide gload / gstore).
template <class P, class Op, int MAXE, bool CAN_FG, bool CAN_TG>
GF_DEV void run_stages(const LineView<typename P::cpx> &s, const KArgs &a, const LineCtx &c,
                       bool cj_first, bool first_g, bool last_g) {
  using TW = typename P::tw_t;
  typename P::cpx v[MAXE];
  const LineProg &lp = a.lp;
  if (lp.nst == 0) {  // length-1 line: the transform is the identity
    if (c.t == 0 && c.valid) {
      typename P::cpx x;
      if constexpr (CAN_FG) {
        if (first_g) x = Op::template gload<P>(a, c, 0);
        else x = s[0];
      } else {
        x = s[0];
      }
      if (cj_first) x.y = -x.y;
      if constexpr (CAN_TG) {
        if (last_g) Op::template gstore<P>(a, c, 0, x);
        else s[0] = x;
      } else {
        s[0] = x;
      }
    }
    __syncthreads();
    return;
  }
  for (int si = 0; si < lp.nst; si++) {
    const int R = lp.radix[si];
    const int ns = lp.ns[si];
    const FastDiv nsd = lp.nsdiv[si];
    const TW *tw = (const TW *)lp.tw + lp.twoff[si];
    const bool cj = cj_first && si == 0;
    const bool fg = first_g && si == 0;
    const bool tg = last_g && si == lp.nst - 1;
    if constexpr (CAN_FG && CAN_TG) {
      if (fg && tg) { stage_sw<P, Op, MAXE, true, true>(R, v, s, a, c, ns, nsd, tw, cj); continue; }
    }
    if constexpr (CAN_FG) {
      if (fg) { stage_sw<P, Op, MAXE, true, false>(R, v, s, a, c, ns, nsd, tw, cj); continue; }
    }
    if constexpr (CAN_TG) {
      if (tg) { stage_sw<P, Op, MAXE, false, true>(R, v, s, a, c, ns, nsd, tw, cj); continue; }
    }
    stage_sw<P, Op, MAXE, false, false>(R, v, s, a, c, ns, nsd, tw, cj);
  }
}

// ---------------------------------------------------------------------------
// Tile loops.  f(l, i, off) is called for local line l, element i (< len),
// with off the element offset of (line, i) on the side.  Rows walk along
// lines; columns walk across lines so consecutive threads touch consecutive
// lines.
// ---------------------------------------------------------------------------
template <class F>
GF_DEV void tile_loop(const Side &sd, int lpc, int len, FastDiv ldiv, FastDiv lpcdiv,
                      long long line0, long long nlines, F f) {
  const int tl = (int)lpcdiv.div((uint32_t)blockDim.x);  // threads per line here
  if ((sd.stride == 1 || lpc == 1) && tl < 8) {
    // short lines: walk the tile element by element so a warp spans lines
    const int total = lpc * len;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      uint32_t l, i;
      ldiv.divmod((uint32_t)e, l, i);
      const long long gl = line0 + l;
      if (gl < nlines) f((int)l, (int)i, line_off(sd, (uint32_t)gl) + (long long)i * sd.stride);
    }
    return;
  }
  // each thread keeps one line: its offset is computed once, the elements
  // step by the threads per line (along the line in row mode, so a warp
  // reads one contiguous run; across lines in column mode, so consecutive
  // threads touch consecutive lines)
  if ((int)threadIdx.x >= tl * lpc) return;
  uint32_t l, i0;
  if (sd.stride == 1 || lpc == 1) {
    l = threadIdx.x / (uint32_t)tl;
    i0 = threadIdx.x - l * (uint32_t)tl;
  } else {
    lpcdiv.divmod(threadIdx.x, i0, l);
  }
  const long long gl = line0 + l;
  if (gl >= nlines) return;
  const long long st = sd.stride;
  long long off = line_off(sd, (uint32_t)gl) + (long long)i0 * st;
  const long long dst = (long long)tl * st;
  for (int i = (int)i0; i < len; i += tl, off += dst) f((int)l, i, off);
}

// A loop over the tile's elements in shared memory only (no global side):
// every (line, element) pair once, each thread on one line, consecutive
// threads on consecutive elements (row layout) or consecutive lines (column
// layout) so shared-memory accesses stay conflict-free.
template <class F>
GF_DEV void smem_loop(const KArgs &a, int len, F f) {
  const int lpc = a.lpc;
  const int tl = (int)a.lpcdiv.div((uint32_t)blockDim.x);
  if ((int)threadIdx.x >= tl * lpc) return;
  uint32_t l, i0;
  if (a.flags & GF_COLMAP) {
    a.lpcdiv.divmod(threadIdx.x, i0, l);
  } else {
    l = threadIdx.x / (uint32_t)tl;
    i0 = threadIdx.x - l * (uint32_t)tl;
  }
  for (int i = (int)i0; i < len; i += tl) f((int)l, i);
}

// ---------------------------------------------------------------------------
// Compile-time schedules.  For the hot lengths the radix list, the threads
// per line and the lines per CTA are template parameters: every stage is
// straight-line code with constant strides, so divisions become shifts, the
// butterfly guards vanish, and the kernel body is only as long as its own
// stages (the run-time schedule kernel carries every radix and thrashes the
// instruction cache).  The twiddle table layout is the run-time one.
// ---------------------------------------------------------------------------
template <int... Rs> struct Sched {};

template <int N, int T, int R> constexpr int ct_per() { return ((N / R) + T - 1) / T; }
template <int N, int T> constexpr int ct_maxe() { return 0; }
template <int N, int T, int R, int... Rs> constexpr int ct_maxe_r() {
  constexpr int here = ct_per<N, T, R>() * R;
  if constexpr (sizeof...(Rs) == 0) return here;
  else {
    constexpr int rest = ct_maxe_r<N, T, Rs...>();
    return here > rest ? here : rest;
  }
}

// Shared-memory slot of element i of a line at base b with element step STEP
// (1 in row layout, the lines per CTA in column layout).  For index runs
// i + r*D with D a multiple of 16 the padded slots are spad(i) + r*(D + D/16),
// so a butterfly's loads and stores share one base address and immediate
// offsets.
template <int STEP, class C> GF_DEV C &slot(C *b, int i) { return b[spad(i) * STEP]; }

// FP64 twiddles of one radix-4/8/16 butterfly from one to three table
// entries.  Plane r-1 of a stage's table holds W^(k r); the other powers are
// products of exactly rounded entries (w^2 = w*w, w^3 = w^2*w, ...: at most
// three products deep, a few ulp), so a butterfly makes one load (three for
// radix 16) where it made R-1.  Each table read is an L1/L2 round trip after
// the stage's barrier; the products are FP64 work, which the line kernels
// have spare.  Measured on the 1024-point FP64 column pass of 4 images:
// 20.2 -> 18.7 us.
template <class P, int R> constexpr bool tw_pow() {
  return std::is_same<P, PrecF64>::value && (R == 4 || R == 8 || R == 16);
}
template <int R> GF_DEV void tw_apply_pow(double2 *x, const double2 *tw, int ns, int k) {
  const double2 w1 = ld_keep(&tw[k]);
  const double2 w2 = cmul(w1, w1), w3 = cmul(w2, w1);
  x[1] = cmul(x[1], w1);
  x[2] = cmul(x[2], w2);
  x[3] = cmul(x[3], w3);
  if constexpr (R == 8) {
    const double2 w4 = cmul(w2, w2);
    x[4] = cmul(x[4], w4);
    x[5] = cmul(x[5], cmul(w4, w1));
    x[6] = cmul(x[6], cmul(w4, w2));
    x[7] = cmul(x[7], cmul(w4, w3));
  } else if constexpr (R == 16) {
    const double2 w4 = ld_keep(&tw[3 * ns + k]), w8 = ld_keep(&tw[7 * ns + k]);
    const double2 w12 = cmul(w8, w4);
    x[4] = cmul(x[4], w4);
    x[8] = cmul(x[8], w8);
    x[12] = cmul(x[12], w12);
#pragma unroll
    for (int r = 1; r < 4; r++) {
      const double2 wr = r == 1 ? w1 : (r == 2 ? w2 : w3);
      x[4 + r] = cmul(x[4 + r], cmul(w4, wr));
      x[8 + r] = cmul(x[8 + r], cmul(w8, wr));
      x[12 + r] = cmul(x[12 + r], cmul(w12, wr));
    }
  }
}

// The barrier between a stage's loads and its stores: the whole CTA, or (in
// warp-specialised kernels) only the warps that work on the tile.
struct CtaBar {
  static GF_DEV void sync() { __syncthreads(); }
};

// GUARD: some threads of the block sit out the butterflies (c.t beyond the
// line); every thread still reaches the barriers.  LAND: the inputs come from
// an unpadded copy of the line at lb (element i at lb[i * STEP], as a bulk
// copy lands it) instead of the padded layout; the outputs go to the padded
// layout at sb (the stage reads everything before its barrier, so lb and sb
// may overlap).
template <class P, class Op, int N, int T, int NS, int R, int E, bool FG, bool TG, int STEP, bool GUARD,
          class BAR = CtaBar, bool LAND = false>
GF_DEV void stage_ct(typename P::cpx (&v)[E], typename P::cpx *sb, const KArgs &a, const LineCtx &c,
                     const typename P::tw_t *tw, const float2 *twh, bool cj,
                     const typename P::cpx *lb = nullptr) {
  using C = typename P::cpx;
  constexpr int NB = N / R;
  constexpr int PER = (NB + T - 1) / T;
  constexpr bool EXACT = (NB % T) == 0 && !GUARD;
#pragma unroll
  for (int b = 0; b < PER; b++) {
    const int j = c.t + b * T;
    if (EXACT || j < NB) {
      if constexpr (LAND) {
        const C *p = lb + j * STEP;
#pragma unroll
        for (int r = 0; r < R; r++) {
          C x = p[r * NB * STEP];
          if (cj) x.y = -x.y;
          v[b * R + r] = x;
        }
      } else if constexpr (!FG && NB % 16 == 0) {
        const C *p = &slot<STEP>(sb, j);
#pragma unroll
        for (int r = 0; r < R; r++) {
          C x = p[r * (NB + NB / 16) * STEP];
          if (cj) x.y = -x.y;
          v[b * R + r] = x;
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; r++) {
          C x;
          if constexpr (FG) x = Op::template gload<P>(a, c, j + r * NB);
          else x = slot<STEP>(sb, j + r * NB);
          if (cj) x.y = -x.y;
          v[b * R + r] = x;
        }
      }
    }
  }
  if constexpr (!FG) BAR::sync();
#pragma unroll
  for (int b = 0; b < PER; b++) {
    const int j = c.t + b * T;
    if (EXACT || j < NB) {
      const int q = j / NS, k = j % NS;
      if constexpr (NS > 1) {
        if constexpr (tw_pow<P, R>()) {
          tw_apply_pow<R>(&v[b * R], tw, NS, k);
        } else if constexpr (short_tw<P, N>()) {
#pragma unroll
          for (int r = 1; r < R; r++) v[b * R + r] = cmul(v[b * R + r], ld_keep(&twh[(r - 1) * NS + k]));
        } else {
#pragma unroll
          for (int r = 1; r < R; r++)
            v[b * R + r] = twmul(v[b * R + r], ld_keep(&tw[(r - 1) * NS + k]));
        }
      }
      Dft<R, C>::run(&v[b * R]);
      const int base = q * NS * R + k;
      if constexpr (TG) {
#pragma unroll
        for (int r = 0; r < R; r++) Op::template gstore<P>(a, c, base + r * NS, v[b * R + r]);
      } else if constexpr (NS % 16 == 0) {
        C *p = &slot<STEP>(sb, base);
#pragma unroll
        for (int r = 0; r < R; r++) p[r * (NS + NS / 16) * STEP] = v[b * R + r];
      } else {
#pragma unroll
        for (int r = 0; r < R; r++) slot<STEP>(sb, base + r * NS) = v[b * R + r];
      }
    }
  }
  if constexpr (!TG) BAR::sync();
}

template <class P, class Op, int N, int T, int NS, int TO, int E, bool CAN_FG, bool CAN_TG, int STEP, bool GUARD,
          class BAR, bool LAND, int R, int... Rs>
GF_DEV void stages_ct(typename P::cpx (&v)[E], typename P::cpx *sb, const KArgs &a, const LineCtx &c,
                      bool cj_first, bool fg, bool tg, const typename P::cpx *lb) {
  using TW = typename P::tw_t;
  constexpr bool FIRST = NS == 1;
  constexpr bool LAST = sizeof...(Rs) == 0;
  const TW *tw = (const TW *)a.lp.tw + TO;
  const float2 *twh = short_tw<P, N>() ? (const float2 *)a.lp.tw_hi + TO : nullptr;
  const bool cj = FIRST && cj_first;
  constexpr bool F_OK = FIRST && CAN_FG;
  constexpr bool T_OK = LAST && CAN_TG;
  if constexpr (FIRST && LAND) {
    // first stage from the landing copy (never direct from global memory)
    if constexpr (T_OK) {
      if (tg) stage_ct<P, Op, N, T, NS, R, E, false, true, STEP, GUARD, BAR, true>(v, sb, a, c, tw, twh, cj, lb);
      else stage_ct<P, Op, N, T, NS, R, E, false, false, STEP, GUARD, BAR, true>(v, sb, a, c, tw, twh, cj, lb);
    } else {
      stage_ct<P, Op, N, T, NS, R, E, false, false, STEP, GUARD, BAR, true>(v, sb, a, c, tw, twh, cj, lb);
    }
  } else if constexpr (F_OK && T_OK) {
    if (fg && tg) stage_ct<P, Op, N, T, NS, R, E, true, true, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
    else if (fg) stage_ct<P, Op, N, T, NS, R, E, true, false, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
    else if (tg) stage_ct<P, Op, N, T, NS, R, E, false, true, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
    else stage_ct<P, Op, N, T, NS, R, E, false, false, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
  } else if constexpr (F_OK) {
    if (fg) stage_ct<P, Op, N, T, NS, R, E, true, false, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
    else stage_ct<P, Op, N, T, NS, R, E, false, false, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
  } else if constexpr (T_OK) {
    if (tg) stage_ct<P, Op, N, T, NS, R, E, false, true, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
    else stage_ct<P, Op, N, T, NS, R, E, false, false, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
  } else {
    stage_ct<P, Op, N, T, NS, R, E, false, false, STEP, GUARD, BAR>(v, sb, a, c, tw, twh, cj);
  }
  if constexpr (!LAST)
    stages_ct<P, Op, N, T, NS * R, TO + NS * (R - 1), E, CAN_FG, CAN_TG, STEP, GUARD, BAR, LAND, Rs...>(
        v, sb, a, c, cj_first, fg, tg, lb);
}

// Runs the compiled schedule on the line at shared-memory base sb; STEP is
// the element step of the layout (1: row layout, LPC: column layout).  BAR is
// the stages' barrier; LAND makes the first stage read the unpadded landing
// copy at lb.
template <class P, class Op, int N, int T, bool CAN_FG, bool CAN_TG, int STEP, bool GUARD = false,
          class BAR = CtaBar, bool LAND = false, int... Rs>
GF_DEV void run_stages_ct(Sched<Rs...>, typename P::cpx *sb, const KArgs &a, const LineCtx &c, bool cj_first,
                          bool fg, bool tg, const typename P::cpx *lb = nullptr) {
  constexpr int E = ct_maxe_r<N, T, Rs...>();
  typename P::cpx v[E];
  stages_ct<P, Op, N, T, 1, 0, E, CAN_FG, CAN_TG, STEP, GUARD, BAR, LAND, Rs...>(v, sb, a, c, cj_first, fg, tg, lb);
}

}  // namespace gf
