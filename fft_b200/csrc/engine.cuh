// engine.cuh -- the B200 line-FFT engine.
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
// Each stage is register-staged: every thread first loads all of its
// butterflies' inputs from shared memory, the CTA synchronises, then each
// thread computes and writes its outputs back over the same buffer.  One
// buffer per line suffices, which doubles the longest single-CTA length.
//
// Global memory is touched only by the tile loops (prologue and epilogue):
// the whole CTA cooperates over lpc x n elements, walking either along lines
// (rows, unit stride) or across lines (columns of a row-major array), so both
// sides are coalesced whatever the transform's axis.
#pragma once
#include "codelets.cuh"

#define GF_MAXST 24

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
};

// Addressing of one side of a batched, strided set of lines (in elements).
// line l, element i:  (l / lpb) * dist_b + (l % lpb) * dist_l + i * stride.
struct Side {
  void *ptr;
  long long dist_b, dist_l, stride;
  FastDiv lpb;
};

GF_DEV long long line_off(const Side &s, uint32_t l) {
  uint32_t b, r;
  s.lpb.divmod(l, b, r);
  return (long long)b * s.dist_b + (long long)r * s.dist_l;
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
  FastDiv ndiv;      // divide by the tile's row length (n, or bins for untangle)
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
// Stockham stage on shared memory.
// ---------------------------------------------------------------------------
template <class P, int R, int MAXE>
GF_DEV void stage(typename P::cpx (&v)[MAXE], typename P::cpx *s, int n, int T, int ns,
                  FastDiv nsd, const typename P::tw_t *tw, int t, bool cj) {
  using C = typename P::cpx;
  constexpr int NB = MAXE / R;
  const int nb = n / R;
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int j = t + b * T;
    if (j < nb) {
#pragma unroll
      for (int r = 0; r < R; r++) {
        C x = s[spad(j + r * nb)];
        if (cj) x.y = -x.y;
        v[b * R + r] = x;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int j = t + b * T;
    if (j < nb) {
      uint32_t q, k;
      nsd.divmod((uint32_t)j, q, k);
      if (ns > 1) {
#pragma unroll
        for (int r = 1; r < R; r++)
          v[b * R + r] = twmul(v[b * R + r], __ldg(&tw[(r - 1) * ns + k]));
      }
      Dft<R, C>::run(&v[b * R]);
      const int base = (int)q * ns * R + (int)k;
#pragma unroll
      for (int r = 0; r < R; r++) s[spad(base + r * ns)] = v[b * R + r];
    }
  }
  __syncthreads();
}

// Runs every stage of lp on the line buffer s.  All threads of the CTA call
// this (stages contain CTA barriers).  One register array serves every radix:
// giving each radix case its own array makes ptxas allocate the switch
// alternatives jointly and spill.  cj_first conjugates the inputs of the
// first stage (or, for a stage-less line of length 1, the element itself).
template <class P, int MAXE>
GF_DEV void run_stages(typename P::cpx *s, const LineProg &lp, int t, bool cj_first) {
  using TW = typename P::tw_t;
  typename P::cpx v[MAXE];
  const int n = lp.n, T = lp.T;
  if (lp.nst == 0) {
    if (cj_first && t == 0) s[0].y = -s[0].y;
    __syncthreads();
    return;
  }
  for (int si = 0; si < lp.nst; si++) {
    const int ns = lp.ns[si];
    const FastDiv nsd = lp.nsdiv[si];
    const TW *tw = (const TW *)lp.tw + lp.twoff[si];
    const bool cj = cj_first && si == 0;
    switch (lp.radix[si]) {
      case 2: stage<P, 2, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      case 3: stage<P, 3, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      case 4: stage<P, 4, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      case 5: stage<P, 5, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      case 7: stage<P, 7, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      case 8: stage<P, 8, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      case 11: stage<P, 11, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      case 13: stage<P, 13, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      case 16: stage<P, 16, MAXE>(v, s, n, T, ns, nsd, tw, t, cj); break;
      default: break;
    }
  }
}

// ---------------------------------------------------------------------------
// Tile loops.  f(l, i, off) is called for local line l, element i, with off the
// element offset of (line, i) on the side.  Rows walk along lines; columns walk
// across lines so consecutive threads touch consecutive lines.
// ---------------------------------------------------------------------------
template <class F>
GF_DEV void tile_loop(const Side &sd, int lpc, int len, FastDiv ldiv, FastDiv lpcdiv,
                      long long line0, long long nlines, F f) {
  const int total = lpc * len;
  if (sd.stride == 1 || lpc == 1) {
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      uint32_t l, i;
      ldiv.divmod((uint32_t)e, l, i);
      const long long gl = line0 + l;
      if (gl < nlines) f((int)l, (int)i, line_off(sd, (uint32_t)gl) + (long long)i * sd.stride);
    }
  } else {
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      uint32_t i, l;
      lpcdiv.divmod((uint32_t)e, i, l);
      const long long gl = line0 + l;
      if (gl < nlines) f((int)l, (int)i, line_off(sd, (uint32_t)gl) + (long long)i * sd.stride);
    }
  }
}

template <class P> GF_DEV typename P::cpx *line_buf(int l, int n) {
  extern __shared__ __align__(16) unsigned char g_smem[];
  return reinterpret_cast<typename P::cpx *>(g_smem) + (size_t)l * spad_size(n);
}
// Two spare complex slots per line after the lpc line buffers.
template <class P> GF_DEV typename P::cpx *line_extra(int l, int n, int lpc) {
  extern __shared__ __align__(16) unsigned char g_smem[];
  return reinterpret_cast<typename P::cpx *>(g_smem) + (size_t)lpc * spad_size(n) + 2 * l;
}

// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async): a tile's loads are all in
// flight before any thread waits, so the prologue is bandwidth- rather than
// latency-bound.  Data that needs arithmetic on arrival (conjugation, chirp,
// window, real-spectrum folding) is copied raw and fixed up in shared memory.
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
// One element of `bytes` (4, 8 or 16).
template <int BYTES> GF_DEV void cp_async_n(void *s, const void *g) {
  if constexpr (BYTES == 16) cp_async16(s, g);
  else if constexpr (BYTES == 8) cp_async8(s, g);
  else cp_async4(s, g);
}

// KArgs::ic bit used by the real-input ops: real pairs are aligned to the
// pair size, so a pair moves as one vector copy.
#define GF_PAIR_ALIGNED 0x40000000

// ---------------------------------------------------------------------------
// Ops.  load() issues the prologue copies (completed by the kernel before
// prep()); prep() runs in-shared-memory fix-ups and ends with a barrier when it
// does anything; store() is the epilogue.  first_conj() asks the first Stockham
// stage to conjugate what it reads (the inverse via conj(DFT(conj x))).
// ---------------------------------------------------------------------------

// Plain complex line: optional conjugation (inverse) and scale.
struct OpC2C {
  static constexpr bool kConv = false;
  static GF_DEV bool first_conj(const KArgs &a) { return a.cj_in; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    const C *in = (const C *)a.in.ptr;
    const int n = a.lp.n;
    tile_loop(a.in, a.lpc, n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      cp_async_n<sizeof(C)>(&line_buf<P>(l, n)[spad(i)], &in[off]);
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    C *out = (C *)a.out.ptr;
    const int n = a.lp.n;
    const Rl sc = (Rl)a.scale;
    const Rl sy = a.cj_out ? -sc : sc;
    tile_loop(a.out, a.lpc, n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      C y = line_buf<P>(l, n)[spad(i)];
      out[off] = mkc(y.x * sc, y.y * sy);
    });
  }
};

// Four-step pass 1 epilogue: element k1 of line n2 (line index within its
// batch) is multiplied by W_N^{n2*k1} from the table aux0 (N entries).
struct OpC2CTwiddle {
  static constexpr bool kConv = false;
  static GF_DEV bool first_conj(const KArgs &a) { return a.cj_in; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    OpC2C::load<P>(a, line0);
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using TW = typename P::tw_t;
    C *out = (C *)a.out.ptr;
    const TW *tw = (const TW *)a.aux0;
    const int n = a.lp.n;
    const long long NN = a.ia;  // full length N
    tile_loop(a.out, a.lpc, n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      const uint32_t gl = (uint32_t)(line0 + l);
      uint32_t b, n2;
      a.out.lpb.divmod(gl, b, n2);
      const long long e = ((long long)n2 * i) % NN;
      C y = line_buf<P>(l, n)[spad(i)];
      out[off] = twmul(y, __ldg(&tw[e]));
    });
  }
};

// Copies the real pair (x[2j], x[2j+1]) of a line into complex slot j.
template <class P>
GF_DEV void load_real_pair(const KArgs &a, typename P::cpx *dst, long long base, long long st) {
  using Rl = typename P::real;
  const Rl *in = (const Rl *)a.in.ptr;
  if (a.ic & GF_PAIR_ALIGNED) {
    cp_async_n<2 * sizeof(Rl)>(dst, &in[base]);
  } else {
    cp_async_n<sizeof(Rl)>(&dst->x, &in[base]);
    cp_async_n<sizeof(Rl)>(&dst->y, &in[base + st]);
  }
}

// Even-length real forward: the 2m reals of a line are read as m complex
// values z[j] = x[2j] + i x[2j+1]; after the m-point FFT the untangle
//   X[k] = (Z[k] + conj Z[m-k])/2 + W_2m^k (Z[k] - conj Z[m-k])/(2i)
// writes bins 0..m (aux0 = W_2m^k table, k = 0..m).  Sides count reals on
// input and complex bins on output.
struct OpR2CPacked {
  static constexpr bool kConv = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    const int m = a.lp.n;
    const long long st = a.in.stride;
    tile_loop(a.in, a.lpc, m, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      // off addresses element j with stride st; the real pair is at 2j, 2j+1
      const long long base = off - (long long)j * st + 2LL * j * st;
      load_real_pair<P>(a, &line_buf<P>(l, m)[spad(j)], base, st);
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    using TW = typename P::tw_t;
    C *out = (C *)a.out.ptr;
    const TW *tw = (const TW *)a.aux0;
    const int m = a.lp.n;
    const int h = m / 2 + 1;  // pair index k = 0..m/2
    const Rl half = (Rl)0.5;
    const long long st = a.out.stride;
    tile_loop(a.out, a.lpc, h, FastDiv((uint32_t)h), a.lpcdiv, line0, a.nlines,
              [&](int l, int k, long long off) {
                const C *s = line_buf<P>(l, m);
                const long long base = off - (long long)k * st;
                if (k == 0) {
                  C z0 = s[spad(0)];
                  out[base] = mkc(z0.x + z0.y, (Rl)0);
                  out[base + (long long)m * st] = mkc(z0.x - z0.y, (Rl)0);
                  return;
                }
                C zk = s[spad(k)], zm = s[spad(m - k)];
                C xe = mkc((zk.x + zm.x) * half, (zk.y - zm.y) * half);
                C xo = mkc((zk.y + zm.y) * half, (zm.x - zk.x) * half);
                C t = twmul(xo, __ldg(&tw[k]));
                out[off] = cadd(xe, t);
                if (m - k != k) out[base + (long long)(m - k) * st] = mkc(xe.x - t.x, t.y - xe.y);
              });
  }
};

GF_DEV double2 cconj_tw(double2 w) { return make_double2(w.x, -w.y); }
GF_DEV float2 cconj_tw(float2 w) { return make_float2(w.x, -w.y); }
GF_DEV float4 cconj_tw(float4 w) { return make_float4(w.x, -w.y, w.z, -w.w); }

// Copies bins 0..min(nb, cnt)-1 of each line raw into slots 0.., zeroing the
// slots of missing bins up to cnt.
template <class P>
GF_DEV void load_bins(const KArgs &a, long long line0, int slots, int cnt, int nb) {
  using C = typename P::cpx;
  using Rl = typename P::real;
  const C *in = (const C *)a.in.ptr;
  tile_loop(a.in, a.lpc, cnt, FastDiv((uint32_t)cnt), a.lpcdiv, line0, a.nlines,
            [&](int l, int k, long long off) {
              C *d = &line_buf<P>(l, slots)[spad(k)];
              if (k < nb) cp_async_n<sizeof(C)>(d, &in[off]);
              else *d = mkc((Rl)0, (Rl)0);
            });
}

// Even-length real inverse: bins 0..m (fewer if ic < m+1: missing bins read
// as zero; imaginary parts of bins 0 and m ignored) are folded back into the
// m-point packed spectrum Z, which is inverse transformed (conjugate trick)
// and unpacked into 2m reals scaled by `scale`.  aux0 = W_2m^k table.
struct OpC2RPacked {
  static constexpr bool kConv = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    const int m = a.lp.n;
    load_bins<P>(a, line0, m, m + 1, a.ic & 0x3fffffff);
  }
  template <class P> static GF_DEV void prep(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    using TW = typename P::tw_t;
    const TW *tw = (const TW *)a.aux0;
    const int m = a.lp.n;
    const int h = m / 2 + 1;
    const Rl half = (Rl)0.5;
    const int total = a.lpc * h;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = e / h, k = e - l * h;
      if (line0 + l >= a.nlines) continue;
      C *s = line_buf<P>(l, m);
      if (k == 0) {
        const Rl x0 = s[spad(0)].x, xm = s[spad(m)].x;
        // Z[0] = ((x0+xm) + i(x0-xm))/2, stored conjugated
        s[spad(0)] = mkc((x0 + xm) * half, -(x0 - xm) * half);
        continue;
      }
      C xk = s[spad(k)], xmk = s[spad(m - k)];
      // xe = (X[k] + conj X[m-k])/2 ; d = (X[k] - conj X[m-k])/2
      C xe = mkc((xk.x + xmk.x) * half, (xk.y - xmk.y) * half);
      C d = mkc((xk.x - xmk.x) * half, (xk.y + xmk.y) * half);
      C xo = twmul(d, cconj_tw(__ldg(&tw[k])));
      // Z[k] = xe + i xo ; Z[m-k] = conj(xe - i xo); stored conjugated
      s[spad(k)] = cconj(mkc(xe.x - xo.y, xe.y + xo.x));
      if (m - k != k) s[spad(m - k)] = cconj(mkc(xe.x + xo.y, -(xe.y - xo.x)));
    }
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    Rl *out = (Rl *)a.out.ptr;
    const int m = a.lp.n;
    const Rl sc = (Rl)a.scale;
    const long long st = a.out.stride;
    tile_loop(a.out, a.lpc, m, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      C y = line_buf<P>(l, m)[spad(j)];
      const long long base = off - (long long)j * st + 2LL * j * st;
      out[base] = y.x * sc;
      out[base + st] = -y.y * sc;
    });
  }
};

// Odd (or any) length real forward through a full complex line: reals are
// copied into the real parts, imaginary parts zeroed; the first n/2+1 bins
// are stored.
struct OpR2CFull {
  static constexpr bool kConv = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using Rl = typename P::real;
    const Rl *in = (const Rl *)a.in.ptr;
    const int n = a.lp.n;
    tile_loop(a.in, a.lpc, n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      typename P::cpx *d = &line_buf<P>(l, n)[spad(i)];
      cp_async_n<sizeof(Rl)>(&d->x, &in[off]);
      d->y = (Rl)0;
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    C *out = (C *)a.out.ptr;
    const int n = a.lp.n;
    const int h = n / 2 + 1;
    tile_loop(a.out, a.lpc, h, FastDiv((uint32_t)h), a.lpcdiv, line0, a.nlines,
              [&](int l, int k, long long off) { out[off] = line_buf<P>(l, n)[spad(k)]; });
  }
};

// Odd (or any) length real inverse through the full Hermitian mirror:
// element i < n/2+1 is bin i, element i > n/2 is conj(bin(n-i)); bins at or
// beyond ic read as zero.  Stored conjugated; the real part is the output.
struct OpC2RFull {
  static constexpr bool kConv = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    const int n = a.lp.n;
    load_bins<P>(a, line0, n, n / 2 + 1, a.ic & 0x3fffffff);
  }
  template <class P> static GF_DEV void prep(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    const int n = a.lp.n;
    const int h = n / 2 + 1;
    const int up = n - h;  // mirrored elements i = h .. n-1
    for (int e = threadIdx.x; e < a.lpc * up; e += blockDim.x) {
      const int l = e / up, i = h + (e - l * up);
      C *s = line_buf<P>(l, n);
      s[spad(i)] = s[spad(n - i)];  // conj(conj(bin(n-i)))
    }
    __syncthreads();
    for (int e = threadIdx.x; e < a.lpc * h; e += blockDim.x) {
      const int l = e / h, i = e - l * h;
      C *s = line_buf<P>(l, n);
      s[spad(i)].y = -s[spad(i)].y;
    }
    __syncthreads();
    (void)line0;
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using Rl = typename P::real;
    Rl *out = (Rl *)a.out.ptr;
    const int n = a.lp.n;
    const Rl sc = (Rl)a.scale;
    tile_loop(a.out, a.lpc, n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      out[off] = line_buf<P>(l, n)[spad(i)].x * sc;
    });
  }
};

}  // namespace gf
