// kernels.cuh -- the line kernel, and the elementwise kernels used by
// multi-pass plans and plan construction (twiddle and spectrum tables).
#pragma once
#include <type_traits>
#include "dispatch.h"
#include "ops.cuh"
#include "rader_ip.cuh"

namespace gf {

// ---------------------------------------------------------------------------
// The line kernel: [tile prologue], stages, [spectrum multiply, stages],
// [tile epilogue].  Threads map along lines (row mode) or across lines
// (GF_COLMAP); the first / last stage read / write global memory directly
// when the op supports it and the host set GF_FIRST_DIRECT / GF_LAST_DIRECT.
// ---------------------------------------------------------------------------
// One tile (lines tile*lpc ..) of a run-time-schedule line op.  Threads at or
// beyond lpc*T (a persistent kernel sized for a larger op) only take part in
// the barriers and the cooperative tile loops.
template <class P, int MAXE, class Op>
GF_DEV void line_body(const KArgs &a, long long tile, bool active) {
  using C = typename P::cpx;
  const long long line0 = tile * a.lpc;
  LineCtx c;
  if (!active) {
    c.l = 0;
    c.t = 1 << 29;  // no butterflies
  } else if (a.flags & GF_COLMAP) {
    c.l = threadIdx.x % a.lpc;
    c.t = threadIdx.x / a.lpc;
  } else {
    c.l = threadIdx.x / a.lp.T;
    c.t = threadIdx.x - c.l * a.lp.T;
  }
  c.line = line0 + c.l;
  c.valid = active && c.line < a.nlines;
  c.ioff = 0;
  c.ooff = 0;
  Op::template load<P>(a, line0);
  cp_async_wait_all();
  __syncthreads();
  Op::template prep<P>(a, line0);
  const LineView<C> s = line_view<C>(a, c.l);
  if constexpr (Op::kConv) {
    run_stages<P, Op, MAXE, false, false>(s, a, c, Op::first_conj(a), false, false);
    Op::template mid<P>(a, line0, false);
    run_stages<P, Op, MAXE, false, false>(s, a, c, false, false, false);
  } else {
    run_stages<P, Op, MAXE, false, false>(s, a, c, Op::first_conj(a), false, false);
  }
  Op::template store<P>(a, line0);
}

// Programmatic dependent launch.  A line kernel launched with programmatic
// stream serialization may be resident before the stream's previous kernel
// has finished: it first waits until that grid has completed and its writes
// are visible (griddepcontrol.wait; returns at once for a kernel launched
// without the attribute, whose predecessors have already completed).  With
// GF_PDL_TRIGGER it then allows the stream's next kernel to be scheduled
// (griddepcontrol.launch_dependents): that kernel's CTAs take SMs as this
// grid's last CTAs retire, and wait in their own griddepcontrol.wait.
GF_DEV void pdl_enter(int flags) {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  if (flags & GF_PDL_TRIGGER) asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// The run-time-schedule kernel always uses the tile prologue / epilogue:
// direct stages would multiply its (already long) body by four.
template <class P, int MAXE, class Op>
__global__ void __launch_bounds__(512, 1) k_line(const KArgs a) {
  pdl_enter(a.flags);
  line_body<P, MAXE, Op>(a, blockIdx.x, true);
}

// ---------------------------------------------------------------------------
// Persistent multi-phase kernel (uneven batches).  A phase is one line op over
// ntiles tiles; items (phase, tile) are numbered phase by phase and claimed
// from a global counter.  A phase with a prerequisite waits until every tile
// of that phase is done: its items come later in the numbering, so the
// prerequisite's items were claimed by running CTAs that never wait on later
// items, and the wait ends.  Each wait is bounded: past spin_limit polls the
// CTA sets *err (results are then invalid and the host reports a timeout).
// Once *err is set, every CTA stops waiting and skips the remaining items'
// transforms (still counting them done), so the kernel drains at once
// instead of spending spin_limit polls on each later dependent item.
// ---------------------------------------------------------------------------
struct PhaseDesc {
  KArgs a;
  int op;
  int dep;           // prerequisite phase or -1
  long long ntiles;
  long long first;   // number of the phase's first item
};

// A persistent kernel's tile on a compiled schedule (complex group-0 ops with
// the tile prologue and epilogue; uneven phases have no direct stages).
// Threads past the phase's LPC*T threads take part in the barriers only.  Not
// inlined: each body keeps its own register allocation.
template <class P, int N, int T, int LPC, class Op, class S>
__device__ __noinline__ void persist_ct_body(const KArgs &a, long long tile, bool active) {
  using C = typename P::cpx;
  const long long line0 = tile * LPC;
  LineCtx c;
  if (!active) {
    c.l = 0;
    c.t = 1 << 29;  // no butterflies
  } else if (a.flags & GF_COLMAP) {
    c.l = threadIdx.x % LPC;
    c.t = threadIdx.x / LPC;
  } else {
    c.l = threadIdx.x / T;
    c.t = threadIdx.x % T;
  }
  c.line = line0 + c.l;
  c.valid = active && c.line < a.nlines;
  c.ioff = 0;
  c.ooff = 0;
  Op::template load<P>(a, line0);
  cp_async_wait_all();
  __syncthreads();
  Op::template prep<P>(a, line0);
  C *sb = line_view<C>(a, c.l).b;
  if (a.flags & GF_COLMAP)
    run_stages_ct<P, Op, N, T, false, false, LPC, true>(S{}, sb, a, c, Op::first_conj(a), false, false);
  else
    run_stages_ct<P, Op, N, T, false, false, 1, true>(S{}, sb, a, c, Op::first_conj(a), false, false);
  Op::template store<P>(a, line0);
}

// Runs the tile on a compiled schedule when one matches the phase (defined
// beside the list of compiled schedules); false otherwise.
template <class P> GF_DEV bool persist_ct(const KArgs &a, int op, long long tile, bool active);

// One op's run-time-schedule body as its own function (not inlined: the
// persistent kernel calls one per phase, and inlining all of them into one
// body made the register allocator spill).
template <class P, class Op>
__device__ __noinline__ void persist_line_body(const KArgs &a, long long tile, bool active) {
  line_body<P, 16, Op>(a, tile, active);
}

// One signal of an in-shared-memory Rader phase (one line per item; every
// thread of the CTA works on it).
template <class P>
__device__ __noinline__ void persist_rip_body(const KArgs &a, long long line) {
  if (line < a.nlines) rader_ip_line<P>(a, line);
}

template <class P>
GF_DEV void phase_dispatch(const KArgs &a, int op, long long tile, bool active) {
  if ((op == OP_C2C || op == OP_C2C_TW) && persist_ct<P>(a, op, tile, active)) return;
  switch (op) {
    case OP_C2C: persist_line_body<P, OpC2C>(a, tile, active); break;
    case OP_C2C_TW: persist_line_body<P, OpC2CTwiddle>(a, tile, active); break;
    case OP_RADER: persist_line_body<P, OpRader>(a, tile, active); break;
    case OP_BLUE: persist_line_body<P, OpBluestein>(a, tile, active); break;
    case OP_RADER_FS1: persist_line_body<P, OpRaderFS1>(a, tile, active); break;
    case OP_RADER_FS2: persist_line_body<P, OpRaderFS2>(a, tile, active); break;
    case OP_RADER_FS4: persist_line_body<P, OpRaderFS4>(a, tile, active); break;
    case OP_RADER_IP: persist_rip_body<P>(a, tile); break;
    default: break;
  }
}

template <class P>
__global__ void __launch_bounds__(512, 1) k_persist(const PhaseDesc *ph, int nph, long long total,
                                                     unsigned long long *ctr, int *done, int *err,
                                                     long long spin_limit) {
  __shared__ __align__(16) unsigned char sa_raw[sizeof(KArgs)];
  KArgs &sa = *reinterpret_cast<KArgs *>(sa_raw);
  __shared__ long long s_item;
  __shared__ int s_p, s_failed;
  for (;;) {
    if (threadIdx.x == 0) {
      const long long it = (long long)atomicAdd(ctr, 1ull);
      s_item = it;
      s_failed = *((volatile int *)err);
      if (it < total) {
        int lo = 0, hi = nph - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) / 2;
          if (ph[mid].first <= it) lo = mid;
          else hi = mid - 1;
        }
        s_p = lo;
        const int d = ph[lo].dep;
        if (d >= 0 && !s_failed) {
          const int need = (int)ph[d].ntiles;
          long long polls = 0;
          while (*((volatile int *)&done[d]) < need) {
            if (*((volatile int *)err)) {  // another CTA gave up: drain
              s_failed = 1;
              break;
            }
            if (++polls > spin_limit) {
              atomicExch(err, 1);
              s_failed = 1;
              break;
            }
            __nanosleep(128);
          }
          __threadfence();
        }
      }
    }
    __syncthreads();
    const long long item = s_item;
    if (item >= total) break;
    const int p = s_p;
    if (!s_failed) {
      {
        const int *src = reinterpret_cast<const int *>(&ph[p].a);
        int *dst = reinterpret_cast<int *>(&sa);
        for (int i = threadIdx.x; i < (int)(sizeof(KArgs) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
      }
      __syncthreads();
      const bool active = threadIdx.x < sa.lpc * sa.lp.T;
      phase_dispatch<P>(sa, ph[p].op, item - ph[p].first, active);
      __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&done[p], 1);
  }
}

// Whether an op has row-layout fast paths (load_row / prep_row / store_row).
template <class Op, class = void> struct RowFast : std::false_type {};
template <class Op> struct RowFast<Op, std::void_t<decltype(Op::kRowFast)>> : std::bool_constant<Op::kRowFast> {};
template <class Op> constexpr bool row_fast() { return RowFast<Op>::value; }

// ---------------------------------------------------------------------------
// Compile-time-schedule line kernel (hot power-of-two lengths): same phases as
// k_line, with N, T, the lines per CTA and the radix list fixed.  Not used for
// the convolution ops.
// ---------------------------------------------------------------------------
template <class P, int N, int T, int LPC, int MINB, class Op, class S>
__global__ void __launch_bounds__(LPC *T, MINB) k_line_ct(const KArgs a) {
  using C = typename P::cpx;
  pdl_enter(a.flags);
  const long long line0 = (long long)blockIdx.x * LPC;
  LineCtx c;
  if (a.flags & GF_COLMAP) {
    c.l = threadIdx.x % LPC;
    c.t = threadIdx.x / LPC;
  } else {
    c.l = threadIdx.x / T;
    c.t = threadIdx.x % T;
  }
  c.line = line0 + c.l;
  c.valid = c.line < a.nlines;
  c.ioff = c.valid ? line_off(a.in, (uint32_t)c.line) : 0;
  c.ooff = c.valid ? line_off(a.out, (uint32_t)c.line) : 0;
  const bool first_g = Op::kFG && (a.flags & GF_FIRST_DIRECT);
  const bool last_g = Op::kTG && (a.flags & GF_LAST_DIRECT);
  const LineView<C> s = line_view<C>(a, c.l);
  if constexpr (Op::kConv) {
    // convolution ops: forward schedule (first stage from global memory when
    // the layout allows), the op's middle step, the schedule again on
    // conjugated data (last stage to global memory when allowed)
    if (!first_g) {
      Op::template load<P>(a, line0);
      cp_async_wait_all();
      __syncthreads();
      Op::template prep<P>(a, line0);
    }
    if (a.flags & GF_COLMAP) {
      run_stages_ct<P, Op, N, T, Op::kFG, false, LPC>(S{}, s.b, a, c, Op::first_conj(a), first_g, false);
      Op::template mid<P>(a, line0, false);
      run_stages_ct<P, Op, N, T, false, Op::kTG, LPC>(S{}, s.b, a, c, false, false, last_g);
    } else {
      run_stages_ct<P, Op, N, T, Op::kFG, false, 1>(S{}, s.b, a, c, Op::first_conj(a), first_g, false);
      Op::template mid<P>(a, line0, false);
      run_stages_ct<P, Op, N, T, false, Op::kTG, 1>(S{}, s.b, a, c, false, false, last_g);
    }
    if (!last_g) Op::template store<P>(a, line0);
    return;
  }
  if constexpr (row_fast<Op>()) {
    // row layout: prologue and epilogue with the stages' own thread mapping
    if (!(a.flags & GF_COLMAP)) {
      if (!first_g) {
        Op::template load_row<P, N, T>(a, c, line0);
        cp_async_wait_all();
        __syncthreads();
        Op::template prep_row<P, N, T>(a, c, s.b);
      }
      run_stages_ct<P, Op, N, T, Op::kFG, Op::kTG, 1>(S{}, s.b, a, c, Op::first_conj(a), first_g, last_g);
      if (!last_g) Op::template store_row<P, N, T>(a, c, s.b);
      return;
    }
  }
  if (!first_g) {
    Op::template load<P>(a, line0);
    cp_async_wait_all();
    __syncthreads();
    Op::template prep<P>(a, line0);
  }
  if (a.flags & GF_COLMAP)
    run_stages_ct<P, Op, N, T, Op::kFG, Op::kTG, LPC>(S{}, s.b, a, c, Op::first_conj(a), first_g, last_g);
  else
    run_stages_ct<P, Op, N, T, Op::kFG, Op::kTG, 1>(S{}, s.b, a, c, Op::first_conj(a), first_g, last_g);
  if (!last_g) Op::template store<P>(a, line0);
}


// ---------------------------------------------------------------------------
// Persistent, double-buffered variant: each CTA walks tiles (lpc lines)
// blockIdx.x, blockIdx.x + gridDim.x, ...  While a tile is transformed in one
// shared buffer, the asynchronous copies of the CTA's next tile fill the
// other, so global-memory latency overlaps the butterflies.  The first stage
// reads shared memory; the last stage writes global memory directly when the
// op and layout allow.
// ---------------------------------------------------------------------------
GF_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
GF_DEV void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
GF_DEV void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <class P, int N, int T, int LPC, int MINB, class Op, class S>
__global__ void __launch_bounds__(LPC *T, MINB) k_line_pp(const KArgs a) {
  using C = typename P::cpx;
  const long long ntiles = (a.nlines + LPC - 1) / LPC;
  long long tile = blockIdx.x;
  if (tile >= ntiles) return;
  C *bufs[2] = {smem_base<C>(), smem_base<C>() + (size_t)LPC * spad_size(N)};
  LineCtx c;
  if (a.flags & GF_COLMAP) {
    c.l = threadIdx.x % LPC;
    c.t = threadIdx.x / LPC;
  } else {
    c.l = threadIdx.x / T;
    c.t = threadIdx.x % T;
  }
  c.ioff = 0;
  const bool last_g = Op::kTG && (a.flags & GF_LAST_DIRECT);
  Op::template load<P>(a, tile * LPC, bufs[0]);
  cp_async_commit();
  int cur = 0;
  for (; tile < ntiles; tile += gridDim.x) {
    const long long next = tile + gridDim.x;
    if (next < ntiles) {
      Op::template load<P>(a, next * LPC, bufs[cur ^ 1]);
      cp_async_commit();
      cp_async_wait1();
    } else {
      cp_async_wait0();
    }
    __syncthreads();
    const long long line0 = tile * LPC;
    Op::template prep<P>(a, line0, bufs[cur]);
    c.line = line0 + c.l;
    c.valid = c.line < a.nlines;
    c.ooff = c.valid ? line_off(a.out, (uint32_t)c.line) : 0;
    const LineView<C> s = line_view<C>(a, c.l, bufs[cur]);
    if (a.flags & GF_COLMAP)
      run_stages_ct<P, Op, N, T, false, Op::kTG, LPC>(S{}, s.b, a, c, Op::first_conj(a), false, last_g);
    else
      run_stages_ct<P, Op, N, T, false, Op::kTG, 1>(S{}, s.b, a, c, Op::first_conj(a), false, last_g);
    if (!last_g) Op::template store<P>(a, line0, bufs[cur]);
    __syncthreads();
    cur ^= 1;
  }
}

// ===========================================================================
// Table generation (FP64 on the device; exact integer angle reduction).
// ===========================================================================

// exp(-2 pi i e / L) for integer e, 0 <= e < L, reduced to the half period
// (-L/2, L/2] before the FP64 sincospi call so the argument is as small as
// possible.
GF_DEV double2 root_of_unity(long long e, long long L) {
  e %= L;
  if (e < 0) e += L;
  if (2 * e > L) e -= L;
  double s, c;
  sincospi(-2.0 * (double)e / (double)L, &s, &c);
  return make_double2(c, s);
}

GF_DEV void put_tw(double2 *t, long long i, double2 w) { t[i] = w; }
GF_DEV void put_tw(float2 *t, long long i, double2 w) { t[i] = make_float2((float)w.x, (float)w.y); }
GF_DEV void put_tw(float4 *t, long long i, double2 w) {
  const float hx = (float)w.x, hy = (float)w.y;
  t[i] = make_float4(hx, hy, (float)(w.x - (double)hx), (float)(w.y - (double)hy));
}

// Stage twiddles: entry (stage s, plane r-1, k) = W_{Ns R}^{k r}.
template <class TW>
__global__ void k_gen_stage_tw(TW *tw, StageTab st, long long total) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int s = 0;
    while (s + 1 < st.nst && idx >= st.twoff[s + 1]) s++;
    const long long loc = idx - st.twoff[s];
    const long long ns = st.ns[s], R = st.radix[s];
    const long long r = loc / ns + 1, k = loc % ns;
    put_tw(tw, idx, root_of_unity(k * r, ns * R));
  }
}

// W_L^(k step) for k = 0..count-1 (four-step and real-untangle tables).
template <class TW> __global__ void k_gen_roots(TW *tw, long long L, long long count, long long step) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x)
    put_tw(tw, k, root_of_unity(k * step, L));
}

// Scale an FP64 spectrum by s and store it in the precision's spectrum form.
template <class SP> __global__ void k_store_spectrum(SP *dst, const double2 *src, double s, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    put_tw(dst, k, make_double2(src[k].x * s, src[k].y * s));
}

// ===========================================================================
// Elementwise kernels for multi-pass plans (convolutions longer than one CTA,
// and lines that have to be made contiguous first).
// ===========================================================================

// Gathers nlines lines of length len from a Side into a contiguous buffer of
// lines of length ldst (zero beyond len), optionally permuted through perm
// (element k <- perm[k]) and conjugated; x0s (if non-null) receives element 0
// of each line (conjugated likewise).
template <class C>
__global__ void k_gather(C *dst, Side src, long long nlines, int len, int ldst, const int *perm,
                         const typename std::conditional<sizeof(C) == 16, double2, float4>::type *chirp,
                         int cj, C *x0s) {
  const long long total = nlines * ldst;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / ldst;
    const int k = (int)(e - l * ldst);
    C v;
    v.x = 0;
    v.y = 0;
    const long long base = line_off(src, (uint32_t)l);
    if (k < len) {
      const long long idx = perm ? perm[k] : k;
      v = ((const C *)src.ptr)[base + idx * src.stride];
      if (cj) v.y = -v.y;
      if (chirp) v = spmul(v, chirp[k]);
    }
    dst[e] = v;
    if (x0s && k == 0) {
      C x0 = ((const C *)src.ptr)[base];
      if (cj) x0.y = -x0.y;
      x0s[l] = x0;
    }
  }
}

// Pointwise spectrum multiply with conjugation: y = conj(y * B[k]); when dc is
// non-null, dc[l] = x0s[l] + y_before[0] is recorded first (Rader's DC bin).
template <class C, class SP>
__global__ void k_spec_mul(C *y, const SP *B, long long nlines, int len, const C *x0s, C *dc) {
  const long long total = nlines * len;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / len;
    const int k = (int)(e - l * len);
    C v = y[e];
    if (dc && k == 0) dc[l] = cadd(x0s[l], v);
    y[e] = cconj(spmul(v, B[k]));
  }
}

// Rader scatter: out[0] = dc, out[iperm[qi]] = x0 + conj(y[qi + off]).
template <class C>
__global__ void k_rader_scatter(Side dst, const C *y, long long nlines, int p, int cl, int off,
                                const int *iperm, const C *x0s, const C *dc, int cj, double scale) {
  using Rl = decltype(C().x);
  const long long total = nlines * p;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / p;
    const int i = (int)(e - l * p);
    C v;
    long long d;
    if (i == 0) {
      v = dc[l];
      d = 0;
    } else {
      v = cadd(x0s[l], cconj(y[l * cl + (i - 1) + off]));
      d = iperm[i - 1];
    }
    const Rl sc = (Rl)scale;
    v.x *= sc;
    v.y *= cj ? -sc : sc;
    ((C *)dst.ptr)[line_off(dst, (uint32_t)l) + d * dst.stride] = v;
  }
}

// Bluestein unchirp: out[k] = conj(y[k]) * w[k] (k < n), conj/scale on store.
template <class C, class SP>
__global__ void k_blue_unchirp(Side dst, const C *y, long long nlines, int n, int m, const SP *w,
                               int cj, double scale) {
  using Rl = decltype(C().x);
  const long long total = nlines * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / n;
    const int k = (int)(e - l * n);
    C v = spmul(cconj(y[l * m + k]), w[k]);
    const Rl sc = (Rl)scale;
    v.x *= sc;
    v.y *= cj ? -sc : sc;
    ((C *)dst.ptr)[line_off(dst, (uint32_t)l) + (long long)k * dst.stride] = v;
  }
}

// Elementwise 2-D spectral filter on nb spectra (R x K each, contiguous):
// the unfused form of OpFilterCol's middle step, Y = X * H (conj(H) with
// conj_h), optionally saving X and writing the per-image dH terms
// conj(Xsaved) * G * w_k * dsc (w_k = 1 at k = 0 and 2k = cols, else 2).
template <class C>
__global__ void k_filter_ew(C *spec, const C *H, C *saved, C *part, long long nb, long long R, long long K,
                            long long cols, int fl, double dsc) {
  using Rl = decltype(C().x);
  const long long per = R * K, total = nb * per;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long hi = e % per;
    const long long k = hi % K;
    const C x = spec[e];
    if (fl & 2) saved[e] = x;
    if (fl & 4) {
      const Rl w = (Rl)(((k == 0 || 2 * k == cols) ? 1.0 : 2.0) * dsc);
      const C xb = saved[e];
      part[e] = mkc((xb.x * x.x + xb.y * x.y) * w, (xb.x * x.y - xb.y * x.x) * w);
    }
    C h = H[hi];
    if (fl & 1) h.y = -h.y;
    spec[e] = cmul(x, h);
  }
}

// dH[i] = sum over b of part[b * count + i] (a fixed-order sum, so the
// parameter gradient is reproducible run to run).
template <class C>
__global__ void k_sum_batches(C *dst, const C *part, long long count, long long nb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    C acc = part[i];
    for (long long b = 1; b < nb; b++) acc = cadd(acc, part[b * count + i]);
    dst[i] = acc;
  }
}

// Copies contiguous lines back to a Side (the inverse of k_gather without
// permutation), with conjugation and scale.
template <class C>
__global__ void k_scatter(Side dst, const C *src, long long nlines, int len, int cj, double scale) {
  using Rl = decltype(C().x);
  const long long total = nlines * len;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / len;
    const int k = (int)(e - l * len);
    C v = src[e];
    const Rl sc = (Rl)scale;
    v.x *= sc;
    v.y *= cj ? -sc : sc;
    ((C *)dst.ptr)[line_off(dst, (uint32_t)l) + (long long)k * dst.stride] = v;
  }
}

// ---------------------------------------------------------------------------
// Multi-pass real transforms (half or full line longer than one CTA).
// ---------------------------------------------------------------------------

// Untangle of contiguous packed spectra Z (m per line) into bins 0..m of `dst`
// (realplan.go:138-169).
template <class C, class TW>
__global__ void k_untangle(Side dst, const C *Z, long long nlines, int m, const TW *tw, double wsc) {
  using Rl = decltype(C().x);
  const int h = m / 2 + 1;
  const long long total = nlines * h;
  const Rl half = (Rl)0.5;
  // edge-bin weighting of the adjoints: bins 0 and m times wsc, the rest 2 wsc
  const Rl we = wsc != 0.0 ? (Rl)wsc : (Rl)1, wi = wsc != 0.0 ? (Rl)(2.0 * wsc) : (Rl)1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / h;
    const int k = (int)(e - l * h);
    const C *z = Z + l * m;
    C *o = (C *)dst.ptr + line_off(dst, (uint32_t)l);
    const long long st = dst.stride;
    if (k == 0) {
      C z0 = z[0];
      o[0] = mkc((z0.x + z0.y) * we, (Rl)0);
      o[(long long)m * st] = mkc((z0.x - z0.y) * we, (Rl)0);
      continue;
    }
    C zk = z[k], zm = z[m - k];
    C xe = mkc((zk.x + zm.x) * half, (zk.y - zm.y) * half);
    C xo = mkc((zk.y + zm.y) * half, (zm.x - zk.x) * half);
    C t = twmul(xo, tw[k]);
    const C a = cadd(xe, t);
    o[(long long)k * st] = mkc(a.x * wi, a.y * wi);
    if (m - k != k) o[(long long)(m - k) * st] = mkc((xe.x - t.x) * wi, (t.y - xe.y) * wi);
  }
}

GF_DEV double2 conj_tw(double2 w) { return make_double2(w.x, -w.y); }
GF_DEV float2 conj_tw(float2 w) { return make_float2(w.x, -w.y); }
GF_DEV float4 conj_tw(float4 w) { return make_float4(w.x, -w.y, w.z, -w.w); }

// Reverse untangle (realplan.go:235-272) from bins of `src` (nb per line
// available) into conjugated packed spectra Z (m per line, contiguous).
template <class C, class TW>
__global__ void k_reverse_untangle(C *Z, Side src, long long nlines, int m, int nb, const TW *tw,
                                   int halve) {
  using Rl = decltype(C().x);
  const int h = m / 2 + 1;
  const long long total = nlines * h;
  const Rl half = (Rl)0.5;
  const Rl wi = halve ? half : (Rl)1;  // adjoints: interior bins enter halved
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / h;
    const int k = (int)(e - l * h);
    const C *in = (const C *)src.ptr + line_off(src, (uint32_t)l);
    const long long st = src.stride;
    auto bin = [&](int q) -> C {
      if (q >= nb) return mkc((Rl)0, (Rl)0);
      const C v = in[(long long)q * st];
      return (q > 0 && q < m) ? mkc(v.x * wi, v.y * wi) : v;
    };
    C *z = Z + l * m;
    if (k == 0) {
      const Rl x0 = bin(0).x, xm = bin(m).x;
      z[0] = mkc((x0 + xm) * half, -(x0 - xm) * half);
      continue;
    }
    C xk = bin(k), xmk = bin(m - k);
    C xe = mkc((xk.x + xmk.x) * half, (xk.y - xmk.y) * half);
    C d = mkc((xk.x - xmk.x) * half, (xk.y + xmk.y) * half);
    C xo = twmul(d, conj_tw(tw[k]));
    z[k] = cconj(mkc(xe.x - xo.y, xe.y + xo.x));
    if (m - k != k) z[m - k] = cconj(mkc(xe.x + xo.y, -(xe.y - xo.x)));
  }
}

// Real line -> complex line (imaginary 0), contiguous n per line.
template <class C>
__global__ void k_promote(C *dst, Side src, long long nlines, int n) {
  using Rl = decltype(C().x);
  const long long total = nlines * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / n;
    const int i = (int)(e - l * n);
    dst[e] = mkc(((const Rl *)src.ptr)[line_off(src, (uint32_t)l) + (long long)i * src.stride], (Rl)0);
  }
}

// Bins 0..n/2 of contiguous complex lines (n per line) -> dst.
template <class C>
__global__ void k_copy_bins(Side dst, const C *src, long long nlines, int n, double wsc) {
  using Rl = decltype(C().x);
  const int h = n / 2 + 1;
  const long long total = nlines * h;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / h;
    const int k = (int)(e - l * h);
    C v = src[l * n + k];
    if (wsc != 0.0) {  // edge-bin weighting of the adjoints
      const Rl w = (Rl)((k == 0 || 2 * k == n) ? wsc : 2.0 * wsc);
      v = mkc(v.x * w, v.y * w);
    }
    ((C *)dst.ptr)[line_off(dst, (uint32_t)l) + (long long)k * dst.stride] = v;
  }
}

// Hermitian mirror (realplan.go:197-206) of bins (nb available) into
// conjugated full lines of length n, contiguous.
template <class C>
__global__ void k_mirror(C *dst, Side src, long long nlines, int n, int nb, int halve) {
  using Rl = decltype(C().x);
  const int h = n / 2 + 1;
  const long long total = nlines * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / n;
    const int i = (int)(e - l * n);
    const C *in = (const C *)src.ptr + line_off(src, (uint32_t)l);
    C v;
    if (i < h) {
      v = i < nb ? in[(long long)i * src.stride] : mkc((Rl)0, (Rl)0);
      v.y = -v.y;
    } else {
      const int q = n - i;
      v = q < nb ? in[(long long)q * src.stride] : mkc((Rl)0, (Rl)0);
    }
    if (halve && i != 0 && 2 * i != n) v = mkc(v.x * (Rl)0.5, v.y * (Rl)0.5);
    dst[e] = v;
  }
}

// Real part of contiguous complex lines times scale -> real dst.
template <class C>
__global__ void k_take_real(Side dst, const C *src, long long nlines, int n, double scale) {
  using Rl = decltype(C().x);
  const long long total = nlines * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / n;
    const int i = (int)(e - l * n);
    ((Rl *)dst.ptr)[line_off(dst, (uint32_t)l) + (long long)i * dst.stride] = src[e].x * (Rl)scale;
  }
}

}  // namespace gf
