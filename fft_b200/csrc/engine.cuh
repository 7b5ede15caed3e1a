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
                  FastDiv nsd, const typename P::tw_t *tw, int t) {
  using C = typename P::cpx;
  constexpr int NB = MAXE / R;
  const int nb = n / R;
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int j = t + b * T;
    if (j < nb) {
#pragma unroll
      for (int r = 0; r < R; r++) v[b * R + r] = s[spad(j + r * nb)];
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
// alternatives jointly and spill.
template <class P, int MAXE>
GF_DEV void run_stages(typename P::cpx *s, const LineProg &lp, int t) {
  using TW = typename P::tw_t;
  typename P::cpx v[MAXE];
  const int n = lp.n, T = lp.T;
  for (int si = 0; si < lp.nst; si++) {
    const int ns = lp.ns[si];
    const FastDiv nsd = lp.nsdiv[si];
    const TW *tw = (const TW *)lp.tw + lp.twoff[si];
    switch (lp.radix[si]) {
      case 2: stage<P, 2, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
      case 3: stage<P, 3, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
      case 4: stage<P, 4, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
      case 5: stage<P, 5, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
      case 7: stage<P, 7, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
      case 8: stage<P, 8, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
      case 11: stage<P, 11, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
      case 13: stage<P, 13, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
      case 16: stage<P, 16, MAXE>(v, s, n, T, ns, nsd, tw, t); break;
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
// Ops: prologue (global -> smem) and epilogue (smem -> global).
// ---------------------------------------------------------------------------

// Plain complex line: optional conjugation (inverse) and scale.
struct OpC2C {
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    const C *in = (const C *)a.in.ptr;
    const int n = a.lp.n;
    const bool cj = a.cj_in;
    tile_loop(a.in, a.lpc, n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      C x = in[off];
      if (cj) x.y = -x.y;
      line_buf<P>(l, n)[spad(i)] = x;
    });
  }
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
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    OpC2C::load<P>(a, line0);
  }
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

// Even-length real forward: the 2m reals of a line are read as m complex
// values z[j] = x[2j] + i x[2j+1]; after the m-point FFT the untangle
//   X[k] = (Z[k] + conj Z[m-k])/2 + W_2m^k (Z[k] - conj Z[m-k])/(2i)
// writes bins 0..m (aux0 = W_2m^k table, k = 0..m).  Sides count reals on
// input and complex bins on output.
struct OpR2CPacked {
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    const Rl *in = (const Rl *)a.in.ptr;
    const int m = a.lp.n;
    const long long st = a.in.stride;
    tile_loop(a.in, a.lpc, m, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      // off addresses element j with stride st; the real pair is at 2j, 2j+1
      const long long base = off - (long long)j * st + 2LL * j * st;
      line_buf<P>(l, m)[spad(j)] = mkc(in[base], in[base + st]);
    });
  }
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

// Even-length real inverse: bins 0..m (fewer if ic < m+1: missing bins read
// as zero; imaginary parts of bins 0 and m ignored) are folded back into the
// m-point packed spectrum Z, which is inverse transformed (conjugate trick)
// and unpacked into 2m reals scaled by `scale`.  aux0 = W_2m^k table.
struct OpC2RPacked {
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    using TW = typename P::tw_t;
    const C *in = (const C *)a.in.ptr;
    const TW *tw = (const TW *)a.aux0;
    const int m = a.lp.n;
    const int nb = a.ic;  // bins available per line
    const int h = m / 2 + 1;
    const Rl half = (Rl)0.5;
    const long long st = a.in.stride;
    tile_loop(a.in, a.lpc, h, FastDiv((uint32_t)h), a.lpcdiv, line0, a.nlines,
              [&](int l, int k, long long off) {
                C *s = line_buf<P>(l, m);
                const long long base = off - (long long)k * st;
                auto bin = [&](int q) -> C {
                  return q < nb ? in[base + (long long)q * st] : mkc((Rl)0, (Rl)0);
                };
                if (k == 0) {
                  const Rl x0 = bin(0).x, xm = bin(m).x;
                  // Z[0] = ((x0+xm) + i(x0-xm))/2, stored conjugated
                  s[spad(0)] = mkc((x0 + xm) * half, -(x0 - xm) * half);
                  return;
                }
                C xk = bin(k), xmk = bin(m - k);
                // xe = (X[k] + conj X[m-k])/2 ; d = (X[k] - conj X[m-k])/2
                C xe = mkc((xk.x + xmk.x) * half, (xk.y - xmk.y) * half);
                C d = mkc((xk.x - xmk.x) * half, (xk.y + xmk.y) * half);
                C xo = twmul(d, cconj_tw(__ldg(&tw[k])));
                // Z[k] = xe + i xo ; Z[m-k] = conj(xe - i xo); store conjugates
                C zk = mkc(xe.x - xo.y, xe.y + xo.x);
                s[spad(k)] = cconj(zk);
                if (m - k != k) {
                  C zmk = mkc(xe.x + xo.y, -(xe.y - xo.x));
                  s[spad(m - k)] = cconj(zmk);
                }
              });
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
  static GF_DEV double2 cconj_tw(double2 w) { return make_double2(w.x, -w.y); }
  static GF_DEV float2 cconj_tw(float2 w) { return make_float2(w.x, -w.y); }
  static GF_DEV float4 cconj_tw(float4 w) { return make_float4(w.x, -w.y, w.z, -w.w); }
};

// Odd (or any) length real forward through a full complex line: reals are
// promoted on load, the first n/2+1 bins are stored.
struct OpR2CFull {
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using Rl = typename P::real;
    const Rl *in = (const Rl *)a.in.ptr;
    const int n = a.lp.n;
    tile_loop(a.in, a.lpc, n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      line_buf<P>(l, n)[spad(i)] = mkc(in[off], (Rl)0);
    });
  }
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
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    const C *in = (const C *)a.in.ptr;
    const int n = a.lp.n;
    const int h = n / 2 + 1;
    const int nb = a.ic;
    const long long st = a.in.stride;
    tile_loop(a.in, a.lpc, n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      const long long base = off - (long long)i * st;
      C v;
      if (i < h) {
        v = i < nb ? in[off] : mkc((Rl)0, (Rl)0);
        v.y = -v.y;  // conjugate for the inverse
      } else {
        const int q = n - i;
        v = q < nb ? in[base + (long long)q * st] : mkc((Rl)0, (Rl)0);  // conj(conj(bin))
      }
      line_buf<P>(l, n)[spad(i)] = v;
    });
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
