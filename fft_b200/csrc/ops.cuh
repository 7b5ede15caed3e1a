// ops.cuh -- what a line kernel reads and writes around the Stockham stages.
//
// Each op provides some of:
//   gload(a, c, i)      element i of the line's input (direct first stage)
//   gstore(a, c, i, v)  element i of the line's output (direct last stage)
//   load / prep         tile prologue: asynchronous copies into shared memory
//                       and in-shared-memory fix-ups (when the first stage is
//                       not direct, or the op needs element pairs)
//   store               tile epilogue (when the last stage is not direct)
//   mid                 convolution ops: spectrum multiply between the two FFTs
// kFG / kTG say whether gload / gstore exist; first_conj(a) asks the first
// stage to conjugate its inputs (inverse transforms as conj(DFT(conj x))).
#pragma once
#include "engine.cuh"

// KArgs::ic bit used by the real-input ops: real pairs are aligned to the
// pair size, so a pair moves as one vector access.
#define GF_PAIR_ALIGNED 0x40000000
// KArgs::ic bit of the real ops: real-spectrum edge-bin weighting for the
// adjoints -- forward ops multiply bins 0 < k < n/2 (and k = n/2 for odd n)
// by 2, inverse ops divide them by 2 as they are read.
#define GF_EDGE_WEIGHT 0x20000000
// KArgs::ic bit of the packed real ops: the spectrum side is the tiled
// intermediate of a rank-2 real transform (TiledPos below; ib = rows per
// image, the side's Side is the identity, line_off(line) = line).
#define GF_TILED 0x10000000
#define GF_IC_MASK 0x0fffffff

namespace gf {

template <class P> using Cx = typename P::cpx;

GF_DEV double2 cconj_tw(double2 w) { return make_double2(w.x, -w.y); }
GF_DEV float2 cconj_tw(float2 w) { return make_float2(w.x, -w.y); }
GF_DEV float4 cconj_tw(float4 w) { return make_float4(w.x, -w.y, w.z, -w.w); }

// Reads the real pair (x[base], x[base + st]) as one complex value.
template <class P> GF_DEV Cx<P> read_pair(const KArgs &a, long long base, long long st) {
  using Rl = typename P::real;
  const Rl *in = (const Rl *)a.in.ptr;
  if (a.ic & GF_PAIR_ALIGNED) return ld_stream(reinterpret_cast<const Cx<P> *>(&in[base]));
  return mkc(ld_stream(&in[base]), ld_stream(&in[base + st]));
}

// Copies the real pair (x[base], x[base + st]) into a complex slot.
template <class P> GF_DEV void load_real_pair(const KArgs &a, Cx<P> *dst, long long base, long long st) {
  using Rl = typename P::real;
  const Rl *in = (const Rl *)a.in.ptr;
  if (a.ic & GF_PAIR_ALIGNED) {
    cp_async_n<2 * sizeof(Rl)>(dst, &in[base]);
  } else {
    cp_async_n<sizeof(Rl)>(&dst->x, &in[base]);
    cp_async_n<sizeof(Rl)>(&dst->y, &in[base + st]);
  }
}

// The tiled intermediate of a rank-2 real transform (rows x bins half-spectra,
// a block of images).  Column-line Lc = image * bins + bin is stored in
// groups of W = 64 bytes / element size (4 complex128, 8 complex64): element
// (Lc, row) at (Lc / W) * W * rows + W * row + Lc % W.  The W columns a
// column-pass CTA transforms (its lines per CTA) are then one contiguous
// rows x W block -- the image layout gave it one 64-byte row segment per row
// and its loads waited on them -- and the row pass writes 64-byte runs.
template <class P> constexpr int tile_lw() { return sizeof(Cx<P>) == 16 ? 2 : 3; }  // log2 W
template <int LW> struct TiledPos {
  long long lc0, rowW, rowsW;  // first column-line of the row's image, W * row, W * rows
  GF_HD long long at(long long k) const {
    const long long L = lc0 + k;
    return (L >> LW) * rowsW + rowW + (L & ((1 << LW) - 1));
  }
};
template <int LW> GF_HD TiledPos<LW> tiled_pos(long long line, long long rows, long long bins) {
  const long long img = line / rows;
  TiledPos<LW> t;
  t.lc0 = img * bins;
  t.rowW = (line - img * rows) << LW;
  t.rowsW = rows << LW;
  return t;
}

// Walks the tiled elements of the CTA's lines (bins 0..bins-1 of lines
// line0..line0+lpc-1): f(l, k, off) for local line l, bin k and the element
// offset in the tiled buffer.  When the CTA's lines lie in one image (rows
// divisible by the lines per CTA, an even number of them) each warp takes two
// lines x 16 consecutive bins: 32 / (2 W) groups, each a 128-byte contiguous
// piece (two rows of W) of the group's run in global memory, and 16
// consecutive slots of each line in shared memory, so the shared-memory side
// is free of bank conflicts (a warp on four lines x W bins met a four-way
// conflict through the line pitch).  Otherwise element by element.
template <class P, class F> GF_DEV void tiled_loop(const KArgs &a, long long line0, int bins, F f) {
  constexpr int LW = tile_lw<P>(), W = 1 << LW, NG = 32 / (2 * W);
  const int L = a.lpc;
  const long long rows = a.ib;
  const int nw = (int)(blockDim.x >> 5), pairs = L >> 1;
  if (rows % L == 0 && (L & 1) == 0 && (blockDim.x & 31) == 0 && nw % pairs == 0) {
    const TiledPos<LW> tp = tiled_pos<LW>(line0, rows, bins);
    const long long g0 = tp.lc0 >> LW;
    const int ng = (int)(((tp.lc0 + bins - 1) >> LW) - g0 + 1);
    const int lane = (int)(threadIdx.x & 31), warp = (int)(threadIdx.x >> 5);
    const int q = lane & (W - 1), r2 = (lane >> LW) & 1, gsub = lane >> (LW + 1);
    const int l = 2 * (warp % pairs) + r2;
    if (line0 + l >= a.nlines) return;
    const int k0 = (int)((g0 << LW) - tp.lc0) + q;
    const int bstep = nw / pairs;
    // element (group g0 + gi, line l, column q): (g0 + gi) * W * rows + W * (row0 + l) + q
    const long long base = g0 * tp.rowsW + tp.rowW + (l << LW) + q;
    for (int gi = (warp / pairs) * NG + gsub; gi < ng; gi += bstep * NG) {
      const int k = k0 + W * gi;
      if (k < 0 || k >= bins) continue;
      f(l, k, base + (long long)gi * tp.rowsW);
    }
    return;
  }
  for (int e = threadIdx.x; e < L * bins; e += blockDim.x) {
    const int l = e / bins, k = e - l * bins;
    if (line0 + l >= a.nlines) continue;
    f(l, k, tiled_pos<LW>(line0 + l, rows, bins).at(k));
  }
}

// Tiled bins 0..bins-1 (missing bins k >= nb zeroed) of the CTA's lines into
// their line buffers.
template <class P> GF_DEV void load_tiled(const KArgs &a, long long line0, int bins, int nb, void *sb) {
  using C = Cx<P>;
  using Rl = typename P::real;
  const C *in = (const C *)a.in.ptr;
  tiled_loop<P>(a, line0, bins, [&](int l, int k, long long off) {
    C *d = &line_view<C>(a, l, sb)[k];
    if (k < nb) cp_async_n<sizeof(C)>(d, &in[off]);
    else *d = mkc((Rl)0, (Rl)0);
  });
}

// Copies bins 0..min(nb, cnt)-1 of each line raw into slots 0.., zeroing the
// slots of missing bins up to cnt.
template <class P> GF_DEV void load_bins(const KArgs &a, long long line0, int cnt, int nb, void *sb) {
  using C = Cx<P>;
  using Rl = typename P::real;
  const C *in = (const C *)a.in.ptr;
  tile_loop(a.in, a.lpc, cnt, FastDiv((uint32_t)cnt), a.lpcdiv, line0, a.nlines,
            [&](int l, int k, long long off) {
              C *d = &line_view<C>(a, l, sb)[k];
              if (k < nb) cp_async_n<sizeof(C)>(d, &in[off]);
              else *d = mkc((Rl)0, (Rl)0);
            });
}

// ---------------------------------------------------------------------------
// Plain complex line: optional conjugation (inverse) and scale.
// ---------------------------------------------------------------------------
struct OpC2C {
  static constexpr bool kConv = false, kFG = true, kTG = true;
  static GF_DEV bool first_conj(const KArgs &a) { return a.cj_in; }
  // Direct stages: element offsets within a line fit 32 bits (launches whose
  // line extent n * stride does not are given the tile prologue/epilogue).
  template <class P> static GF_DEV Cx<P> gload(const KArgs &a, const LineCtx &c, int i) {
    using Rl = typename P::real;
    if (!c.valid) return mkc((Rl)0, (Rl)0);
    return ld_stream(&((const Cx<P> *)a.in.ptr + c.ioff)[i * (int)a.in.stride]);
  }
  template <class P> static GF_DEV void gstore(const KArgs &a, const LineCtx &c, int i, Cx<P> y) {
    using Rl = typename P::real;
    if (!c.valid) return;
    Cx<P> *o = &((Cx<P> *)a.out.ptr + c.ooff)[i * (int)a.out.stride];
    if (a.scale == 1.0) {  // forward passes: no multiply
      *o = a.cj_out ? mkc(y.x, -y.y) : y;
      return;
    }
    const Rl sc = (Rl)a.scale;
    *o = mkc(y.x * sc, y.y * (a.cj_out ? -sc : sc));
  }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    const C *in = (const C *)a.in.ptr;
    tile_loop(a.in, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      cp_async_n<sizeof(C)>(&line_view<C>(a, l, sb)[i], &in[off]);
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    C *out = (C *)a.out.ptr;
    const Rl sc = (Rl)a.scale;
    const Rl sy = a.cj_out ? -sc : sc;
    tile_loop(a.out, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      C y = line_view<C>(a, l, sb)[i];
      out[off] = mkc(y.x * sc, y.y * sy);
    });
  }
};

// y * W_N^e from a split table (see OpC2CTwiddle): W_N^(e mod 2^sh), then
// W_N^(2^sh floor(e / 2^sh)).
template <class P>
GF_DEV Cx<P> split_tw(Cx<P> y, const typename P::tw_t *t, uint32_t e, int sh) {
  const uint32_t S = 1u << sh;
  return twmul(twmul(y, ld_keep(&t[e & (S - 1)])), ld_keep(&t[S + (e >> sh)]));
}

// Four-step pass 1: element k1 of line n2 (the line's index within its batch)
// is multiplied by W_N^e, e = n2*k1 < N, as W_N^(e mod S) * W_N^(S floor(e/S))
// from the split table aux0 (S = 2^ic entries, then ceil(N/S) entries):
// two small tables that stay in L1 instead of one of N entries read at
// scattered places.  ia = N.
struct OpC2CTwiddle {
  static constexpr bool kConv = false, kFG = true, kTG = true;
  static GF_DEV bool first_conj(const KArgs &a) { return a.cj_in; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &a, const LineCtx &c, int i) {
    return OpC2C::gload<P>(a, c, i);
  }
  template <class P> static GF_DEV Cx<P> tw(const KArgs &a, long long line, int i, Cx<P> y) {
    using TW = typename P::tw_t;
    uint32_t b, n2;
    a.out.lpb.divmod((uint32_t)line, b, n2);
    // n2 < N2 and i < N1, so n2 * i < N1 * N2 = N: the exponent needs no
    // reduction modulo N
    return split_tw<P>(y, (const TW *)a.aux0, n2 * (uint32_t)i, a.ic);
  }
  template <class P> static GF_DEV void gstore(const KArgs &a, const LineCtx &c, int i, Cx<P> y) {
    if (!c.valid) return;
    ((Cx<P> *)a.out.ptr)[c.ooff + (long long)i * a.out.stride] = tw<P>(a, c.line, i, y);
  }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) { OpC2C::load<P>(a, line0, sb); }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    C *out = (C *)a.out.ptr;
    tile_loop(a.out, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      out[off] = tw<P>(a, line0 + l, i, line_view<C>(a, l, sb)[i]);
    });
  }
};

// ---------------------------------------------------------------------------
// Even-length real forward: the 2m reals of a line are read as m complex
// values z[j] = x[2j] + i x[2j+1]; after the m-point FFT the untangle
//   X[k] = (Z[k] + conj Z[m-k])/2 + W_2m^k (Z[k] - conj Z[m-k])/(2i)
// writes bins 0..m (aux0 = W_2m^k table, k = 0..m; FP32-mixed: aux1 = the
// same roots as FP32 hi parts, for short lines).  Sides count reals on
// input and complex bins on output.
// ---------------------------------------------------------------------------
template <class P, class F>
GF_DEV void untangle_tile(const KArgs &a, long long line0, F emit, void *sb) {
  using C = Cx<P>;
  using Rl = typename P::real;
  using TW = typename P::tw_t;
  const TW *tw = (const TW *)a.aux0;
  const int m = a.lp.n;
  const int h = m / 2 + 1;  // pair index k = 0..m/2
  const Rl half = (Rl)0.5;
  tile_loop(a.out, a.lpc, h, FastDiv((uint32_t)h), a.lpcdiv, line0, a.nlines,
            [&](int l, int k, long long off) {
              const LineView<C> s = line_view<C>(a, l, sb);
              const long long base = off - (long long)k * a.out.stride;
              if (k == 0) {
                C z0 = s[0];
                emit(base, 0, mkc(z0.x + z0.y, (Rl)0));
                emit(base, m, mkc(z0.x - z0.y, (Rl)0));
                return;
              }
              C zk = s[k], zm = s[m - k];
              C xe = mkc((zk.x + zm.x) * half, (zk.y - zm.y) * half);
              C xo = mkc((zk.y + zm.y) * half, (zm.x - zk.x) * half);
              C t = twmul(xo, ld_keep(&tw[k]));
              emit(base, k, cadd(xe, t));
              if (m - k != k) emit(base, m - k, mkc(xe.x - t.x, t.y - xe.y));
            });
}

struct OpR2CPacked {
  static constexpr bool kConv = false, kFG = true, kTG = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  // Direct first stage: only launched with unit-stride, pair-aligned rows
  // (GF_PAIR_ALIGNED), so pair j is one vector at element 2j.
  template <class P> static GF_DEV Cx<P> gload(const KArgs &a, const LineCtx &c, int j) {
    using Rl = typename P::real;
    if (!c.valid) return mkc((Rl)0, (Rl)0);
    return ld_stream(reinterpret_cast<const Cx<P> *>((const Rl *)a.in.ptr + c.ioff) + j);
  }
  template <class P> static GF_DEV void gstore(const KArgs &, const LineCtx &, int, Cx<P>) {}
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    const long long st = a.in.stride;
    tile_loop(a.in, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      const long long base = off - (long long)j * st + 2LL * j * st;
      load_real_pair<P>(a, &line_view<Cx<P>>(a, l, sb)[j], base, st);
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using Rl = typename P::real;
    Cx<P> *out = (Cx<P> *)a.out.ptr;
    const long long st = a.out.stride;
    const bool tiled = (a.ic & GF_TILED) != 0;
    const int m = a.lp.n;
    // tiled: the out side is the identity, so base is the line index
    auto at = [&](long long base, int k) {
      return tiled ? tiled_pos<tile_lw<P>()>(base, a.ib, m + 1).at(k) : base + (long long)k * st;
    };
    if (a.ic & GF_EDGE_WEIGHT) {
      const Rl sc = (Rl)a.scale;
      untangle_tile<P>(a, line0, [&](long long base, int k, Cx<P> v) {
        const Rl w = (k == 0 || k == m) ? sc : (Rl)2 * sc;
        out[at(base, k)] = mkc(v.x * w, v.y * w);
      }, sb);
      return;
    }
    untangle_tile<P>(a, line0, [&](long long base, int k, Cx<P> v) { out[at(base, k)] = v; }, sb);
  }
  // Row-layout fast paths for the compiled-schedule kernels (M = lp.n, T
  // threads per line; thread c.t of line c.l, line data at sb).
  static constexpr bool kRowFast = true;
  template <class P, int M, int T> static GF_DEV void load_row(const KArgs &a, const LineCtx &, long long line0) {
    load<P>(a, line0);
  }
  template <class P, int M, int T> static GF_DEV void prep_row(const KArgs &, const LineCtx &, Cx<P> *) {}
  template <class P, int M, int T> static GF_DEV void store_row(const KArgs &a, const LineCtx &c, Cx<P> *sb) {
    using C = Cx<P>;
    using Rl = typename P::real;
    using TW = typename P::tw_t;
    constexpr int H = M / 2 + 1;
    constexpr int IT = (H + T - 1) / T;
    const TW *tw = (const TW *)a.aux0;
    C *out = (C *)a.out.ptr + c.ooff;
    const int st = (int)a.out.stride;
    const Rl half = (Rl)0.5;
    const bool wgt = (a.ic & GF_EDGE_WEIGHT) != 0;
    const Rl sc = (Rl)a.scale;
    const bool tiled = (a.ic & GF_TILED) != 0;
    // bins k and M - k from the packed spectrum's slots k and M - k
    auto untangle = [&](auto emit) {
#pragma unroll
      for (int it = 0; it < IT; it++) {
        const int k = c.t + it * T;
        if (IT * T > H && k >= H) break;
        if (k == 0) {
          const C z0 = sb[0];
          const Rl w = wgt ? sc : (Rl)1;
          emit(0, mkc((z0.x + z0.y) * w, (Rl)0));
          emit(M, mkc((z0.x - z0.y) * w, (Rl)0));
          continue;
        }
        const C zk = sb[spad(k)], zm = sb[spad(M - k)];
        const C xe = mkc((zk.x + zm.x) * half, (zk.y - zm.y) * half);
        const C xo = mkc((zk.y + zm.y) * half, (zm.x - zk.x) * half);
        C t;
        if constexpr (short_tw<P, M>()) t = cmul(xo, ld_keep(&((const float2 *)a.aux1)[k]));
        else t = twmul(xo, ld_keep(&tw[k]));
        C lo = cadd(xe, t), hi = mkc(xe.x - t.x, t.y - xe.y);
        if (wgt) {
          const Rl w2 = (Rl)2 * sc;
          lo = mkc(lo.x * w2, lo.y * w2);
          hi = mkc(hi.x * w2, hi.y * w2);
        }
        emit(k, lo);
        if (M - k != k) emit(M - k, hi);
      }
    };
    if (!c.valid) return;
    if (tiled) {
      const auto tp = tiled_pos<tile_lw<P>()>(c.line, a.ib, M + 1);
      C *tout = (C *)a.out.ptr;
      untangle([&](int kk, C v) { tout[tp.at(kk)] = v; });
    } else {
      untangle([&](int kk, C v) { out[kk * st] = v; });
    }
  }
};

// Even-length real inverse: bins 0..m (fewer if ic < m+1: missing bins read
// as zero; imaginary parts of bins 0 and m ignored) are folded back into the
// m-point packed spectrum Z, which is inverse transformed (conjugate trick)
// and unpacked into 2m reals scaled by `scale`.  aux0 = W_2m^k table
// (FP32-mixed: aux1 = its FP32 hi parts, for short lines).
struct OpC2RPacked {
  static constexpr bool kConv = false, kFG = false, kTG = true;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &, const LineCtx &, int) { return Cx<P>(); }
  template <class P> static GF_DEV void gstore(const KArgs &a, const LineCtx &c, int j, Cx<P> y) {
    using Rl = typename P::real;
    if (!c.valid) return;
    Rl *out = (Rl *)a.out.ptr;
    const Rl sc = (Rl)a.scale;
    // direct last stage: only launched with unit-stride, pair-aligned rows
    reinterpret_cast<Cx<P> *>(out + c.ooff)[j] = mkc(y.x * sc, -y.y * sc);
  }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    const int m = a.lp.n;
    if (a.ic & GF_TILED) load_tiled<P>(a, line0, m + 1, a.ic & GF_IC_MASK, sb);
    else load_bins<P>(a, line0, m + 1, a.ic & GF_IC_MASK, sb);
  }
  template <class P> static GF_DEV void prep(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    using TW = typename P::tw_t;
    const TW *tw = (const TW *)a.aux0;
    const int m = a.lp.n;
    const int h = m / 2 + 1;
    const Rl half = (Rl)0.5;
    smem_loop(a, h, [&](int l, int k) {
      if (line0 + l >= a.nlines) return;
      const LineView<C> s = line_view<C>(a, l, sb);
      if (k == 0) {
        const Rl x0 = s[0].x, xm = s[m].x;
        // Z[0] = ((x0+xm) + i(x0-xm))/2, stored conjugated
        s[0] = mkc((x0 + xm) * half, -(x0 - xm) * half);
        return;
      }
      C xk = s[k], xmk = s[m - k];
      if (a.ic & GF_EDGE_WEIGHT) {  // interior bins enter halved (k = m/2 too)
        xk = mkc(xk.x * half, xk.y * half);
        xmk = mkc(xmk.x * half, xmk.y * half);
      }
      // xe = (X[k] + conj X[m-k])/2 ; d = (X[k] - conj X[m-k])/2
      C xe = mkc((xk.x + xmk.x) * half, (xk.y - xmk.y) * half);
      C d = mkc((xk.x - xmk.x) * half, (xk.y + xmk.y) * half);
      C xo = twmul(d, cconj_tw(ld_keep(&tw[k])));
      // Z[k] = xe + i xo ; Z[m-k] = conj(xe - i xo); stored conjugated
      s[k] = cconj(mkc(xe.x - xo.y, xe.y + xo.x));
      if (m - k != k) s[m - k] = cconj(mkc(xe.x + xo.y, -(xe.y - xo.x)));
    });
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    Rl *out = (Rl *)a.out.ptr;
    const Rl sc = (Rl)a.scale;
    const long long st = a.out.stride;
    tile_loop(a.out, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      C y = line_view<C>(a, l, sb)[j];
      const long long base = off - (long long)j * st + 2LL * j * st;
      out[base] = y.x * sc;
      out[base + st] = -y.y * sc;
    });
  }
  // Row-layout fast paths for the compiled-schedule kernels (M = lp.n).
  static constexpr bool kRowFast = true;
  template <class P, int M, int T> static GF_DEV void load_row(const KArgs &a, const LineCtx &c, long long line0) {
    using C = Cx<P>;
    using Rl = typename P::real;
    constexpr int IT = (M + 1 + T - 1) / T;
    if (a.ic & GF_TILED) {  // the whole CTA copies its lines' tiled runs
      load_tiled<P>(a, line0, M + 1, a.ic & GF_IC_MASK, nullptr);
      return;
    }
    C *d = line_view<C>(a, c.l).b;
    if (!c.valid) return;
    const C *in = (const C *)a.in.ptr + c.ioff;
    const int st = (int)a.in.stride;
    const int nb = a.ic & GF_IC_MASK;
#pragma unroll
    for (int it = 0; it < IT; it++) {
      const int k = c.t + it * T;
      if (IT * T > M + 1 && k > M) break;
      if (k < nb) cp_async_n<sizeof(C)>(&d[spad(k)], &in[k * st]);
      else d[spad(k)] = mkc((Rl)0, (Rl)0);
    }
  }
  template <class P, int M, int T> static GF_DEV void prep_row(const KArgs &a, const LineCtx &c, Cx<P> *s) {
    using C = Cx<P>;
    using Rl = typename P::real;
    using TW = typename P::tw_t;
    constexpr int H = M / 2 + 1;
    constexpr int IT = (H + T - 1) / T;
    const TW *tw = (const TW *)a.aux0;
    const Rl half = (Rl)0.5;
    const bool wgt = (a.ic & GF_EDGE_WEIGHT) != 0;
    if (c.valid) {
#pragma unroll
      for (int it = 0; it < IT; it++) {
        const int k = c.t + it * T;
        if (IT * T > H && k >= H) break;
        if (k == 0) {
          const Rl x0 = s[0].x, xm = s[spad(M)].x;
          s[0] = mkc((x0 + xm) * half, -(x0 - xm) * half);
          continue;
        }
        C xk = s[spad(k)], xmk = s[spad(M - k)];
        if (wgt) {
          xk = mkc(xk.x * half, xk.y * half);
          xmk = mkc(xmk.x * half, xmk.y * half);
        }
        const C xe = mkc((xk.x + xmk.x) * half, (xk.y - xmk.y) * half);
        const C d = mkc((xk.x - xmk.x) * half, (xk.y + xmk.y) * half);
        C xo;
        if constexpr (short_tw<P, M>()) xo = cmul(d, cconj_tw(ld_keep(&((const float2 *)a.aux1)[k])));
        else xo = twmul(d, cconj_tw(ld_keep(&tw[k])));
        s[spad(k)] = cconj(mkc(xe.x - xo.y, xe.y + xo.x));
        if (M - k != k) s[spad(M - k)] = cconj(mkc(xe.x + xo.y, -(xe.y - xo.x)));
      }
    }
    __syncthreads();
  }
  template <class P, int M, int T> static GF_DEV void store_row(const KArgs &a, const LineCtx &, Cx<P> *) {}
};

// Odd (or any) length real forward through a full complex line: reals in the
// real parts, imaginary parts zero; the first n/2+1 bins are stored.
struct OpR2CFull {
  static constexpr bool kConv = false, kFG = true, kTG = true;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &a, const LineCtx &c, int i) {
    using Rl = typename P::real;
    if (!c.valid) return mkc((Rl)0, (Rl)0);
    return mkc(ld_stream(&((const Rl *)a.in.ptr)[c.ioff + (long long)i * a.in.stride]), (Rl)0);
  }
  template <class P> static GF_DEV Cx<P> weigh(const KArgs &a, int k, Cx<P> y) {
    using Rl = typename P::real;
    if (!(a.ic & GF_EDGE_WEIGHT)) return y;
    const int n = a.lp.n;
    const Rl w = (Rl)a.scale * ((k == 0 || 2 * k == n) ? (Rl)1 : (Rl)2);
    return mkc(y.x * w, y.y * w);
  }
  template <class P> static GF_DEV void gstore(const KArgs &a, const LineCtx &c, int i, Cx<P> y) {
    if (!c.valid || i > a.lp.n / 2) return;
    ((Cx<P> *)a.out.ptr)[c.ooff + (long long)i * a.out.stride] = weigh<P>(a, i, y);
  }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    using Rl = typename P::real;
    const Rl *in = (const Rl *)a.in.ptr;
    tile_loop(a.in, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      Cx<P> *d = &line_view<Cx<P>>(a, l, sb)[i];
      cp_async_n<sizeof(Rl)>(&d->x, &in[off]);
      d->y = (Rl)0;
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    C *out = (C *)a.out.ptr;
    const int h = a.lp.n / 2 + 1;
    tile_loop(a.out, a.lpc, h, FastDiv((uint32_t)h), a.lpcdiv, line0, a.nlines,
              [&](int l, int k, long long off) { out[off] = weigh<P>(a, k, line_view<C>(a, l, sb)[k]); });
  }
};

// Odd (or any) length real inverse through the full Hermitian mirror:
// element i < n/2+1 is bin i, element i > n/2 is conj(bin(n-i)); bins at or
// beyond ic read as zero.  Stored conjugated; the real part is the output.
struct OpC2RFull {
  static constexpr bool kConv = false, kFG = false, kTG = true;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &, const LineCtx &, int) { return Cx<P>(); }
  template <class P> static GF_DEV void gstore(const KArgs &a, const LineCtx &c, int i, Cx<P> y) {
    using Rl = typename P::real;
    if (!c.valid) return;
    ((Rl *)a.out.ptr)[c.ooff + (long long)i * a.out.stride] = y.x * (Rl)a.scale;
  }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    load_bins<P>(a, line0, a.lp.n / 2 + 1, a.ic & GF_IC_MASK, sb);
  }
  template <class P> static GF_DEV void prep(const KArgs &a, long long, void *sb = nullptr) {
    using C = Cx<P>;
    const int n = a.lp.n;
    const int h = n / 2 + 1;
    const int up = n - h;  // mirrored elements i = h .. n-1
    if (a.ic & GF_EDGE_WEIGHT) {
      smem_loop(a, h, [&](int l, int i) {
        if (i == 0 || 2 * i == n) return;
        const LineView<C> s = line_view<C>(a, l, sb);
        s[i] = mkc(s[i].x * (typename P::real)0.5, s[i].y * (typename P::real)0.5);
      });
      __syncthreads();
    }
    smem_loop(a, up, [&](int l, int e) {
      const int i = h + e;
      const LineView<C> s = line_view<C>(a, l, sb);
      s[i] = s[n - i];  // conj(conj(bin(n-i)))
    });
    __syncthreads();
    smem_loop(a, h, [&](int l, int i) {
      const LineView<C> s = line_view<C>(a, l, sb);
      s[i].y = -s[i].y;
    });
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using Rl = typename P::real;
    Rl *out = (Rl *)a.out.ptr;
    const Rl sc = (Rl)a.scale;
    tile_loop(a.out, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      out[off] = line_view<Cx<P>>(a, l, sb)[i].x * sc;
    });
  }
};

// ---------------------------------------------------------------------------
// Rader, fused in one CTA (rader.go:129-172 restated for one line):
//   a[k] = x[perm[k]] (k < q = p-1, zero-padded to cl), A = FFT_cl(a),
//   X[0] = x0 + A[0] (= sum of all inputs),
//   conv = IFFT_cl(A * B)  evaluated as conj(FFT_cl(conj(A * B / cl))),
//   X[iperm[qi]] = x0 + conv[qi + off]   (off = 0 cyclic, q padded-linear).
// aux0 = perm (int32, q), aux1 = iperm (int32, q), aux2 = B/cl (sp_t, cl),
// ia = p, ic = off.  lp is the length-cl program; the extra slots of a line
// hold x0 and X[0].
// ---------------------------------------------------------------------------
struct OpRader {
  static constexpr bool kConv = true, kFG = true, kTG = true;
  static GF_DEV bool first_conj(const KArgs &a) { return a.cj_in; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &a, const LineCtx &c, int k) {
    using C = Cx<P>;
    using Rl = typename P::real;
    if (!c.valid) return mkc((Rl)0, (Rl)0);
    const C *in = (const C *)a.in.ptr;
    if (k == 0) {
      C x0 = in[c.ioff];
      if (a.cj_in) x0.y = -x0.y;
      line_extra<C>(a, c.l)[0] = x0;
    }
    const int q = (int)a.ia - 1;
    if (k >= q) return mkc((Rl)0, (Rl)0);
    return in[c.ioff + (long long)__ldg(&((const int *)a.aux0)[k]) * a.in.stride];
  }
  template <class P> static GF_DEV void gstore(const KArgs &a, const LineCtx &c, int i, Cx<P> y) {
    using C = Cx<P>;
    using Rl = typename P::real;
    const int q = (int)a.ia - 1;
    const int qi = i - a.ic;
    if (!c.valid || qi < 0 || qi >= q) return;
    const C v = cadd(line_extra<C>(a, c.l)[0], cconj(y));
    const Rl sc = (Rl)a.scale;
    const long long d = __ldg(&((const int *)a.aux1)[qi]);
    ((C *)a.out.ptr)[c.ooff + d * a.out.stride] = mkc(v.x * sc, v.y * (a.cj_out ? -sc : sc));
  }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    const C *in = (const C *)a.in.ptr;
    const int *perm = (const int *)a.aux0;
    const int cl = a.lp.n;
    const int q = (int)a.ia - 1;
    const long long st = a.in.stride;
    tile_loop(a.in, a.lpc, cl, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int k, long long off) {
      const long long base = off - (long long)k * st;
      C *d = &line_view<C>(a, l, sb)[k];
      if (k < q) cp_async_n<sizeof(C)>(d, &in[base + (long long)__ldg(&perm[k]) * st]);
      else *d = mkc((Rl)0, (Rl)0);
      if (k == 0) {
        C x0 = in[base];
        if (a.cj_in) x0.y = -x0.y;
        line_extra<C>(a, l)[0] = x0;
      }
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void mid(const KArgs &a, long long line0, bool last_g, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    using SP = typename P::sp_t;
    const SP *B = (const SP *)a.aux2;
    const int cl = a.lp.n;
    // X[0] first (reads A[0] before the multiply overwrites it)
    for (int l = threadIdx.x; l < a.lpc; l += blockDim.x) {
      C *ex = line_extra<C>(a, l);
      ex[1] = cadd(ex[0], line_view<C>(a, l, sb)[0]);
      if (last_g && line0 + l < a.nlines) {
        const Rl sc = (Rl)a.scale;
        ((C *)a.out.ptr)[line_off(a.out, (uint32_t)(line0 + l))] =
            mkc(ex[1].x * sc, ex[1].y * (a.cj_out ? -sc : sc));
      }
    }
    __syncthreads();
    const int total = a.lpc * cl;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      uint32_t l, k;
      a.ndiv.divmod((uint32_t)e, l, k);
      const LineView<C> s = line_view<C>(a, (int)l, sb);
      s[k] = cconj(spmul(s[k], __ldg(&B[k])));
    }
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    C *out = (C *)a.out.ptr;
    const int *iperm = (const int *)a.aux1;
    const int p = (int)a.ia;
    const int offc = a.ic;
    const Rl sc = (Rl)a.scale;
    const Rl sy = a.cj_out ? -sc : sc;
    const long long st = a.out.stride;
    tile_loop(a.out, a.lpc, p, FastDiv((uint32_t)p), a.lpcdiv, line0, a.nlines,
              [&](int l, int i, long long off) {
                const long long base = off - (long long)i * st;
                const C *ex = line_extra<C>(a, l);
                C y;
                long long dst;
                if (i == 0) {
                  y = ex[1];
                  dst = 0;
                } else {
                  y = cadd(ex[0], cconj(line_view<C>(a, l, sb)[i - 1 + offc]));
                  dst = __ldg(&iperm[i - 1]);
                }
                out[base + dst * st] = mkc(y.x * sc, y.y * sy);
              });
  }
};

// ---------------------------------------------------------------------------
// Bluestein, fused in one CTA (bluestein.go:67-95 restated for one line):
//   a[j] = x[j] w[j] (j < n, zero-padded to m), conv = IFFT_m(FFT_m(a) * B)
//   with B = FFT_m(b) / m, evaluated as conj(FFT_m(conj(FFT_m(a) * B))),
//   X[k] = conv[k] w[k].
// aux0 = chirp w (sp_t, n), aux2 = B/m (sp_t, m), ia = n.  lp has length m.
// ---------------------------------------------------------------------------
struct OpBluestein {
  static constexpr bool kConv = true, kFG = true, kTG = true;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &a, const LineCtx &c, int j) {
    using C = Cx<P>;
    using Rl = typename P::real;
    using SP = typename P::sp_t;
    if (!c.valid || j >= (int)a.ia) return mkc((Rl)0, (Rl)0);
    C v = ld_stream(&((const C *)a.in.ptr)[c.ioff + (long long)j * a.in.stride]);
    if (a.cj_in) v.y = -v.y;
    return spmul(v, __ldg(&((const SP *)a.aux0)[j]));
  }
  template <class P> static GF_DEV void gstore(const KArgs &a, const LineCtx &c, int k, Cx<P> y) {
    using C = Cx<P>;
    using Rl = typename P::real;
    using SP = typename P::sp_t;
    if (!c.valid || k >= (int)a.ia) return;
    const C v = spmul(cconj(y), __ldg(&((const SP *)a.aux0)[k]));
    const Rl sc = (Rl)a.scale;
    ((C *)a.out.ptr)[c.ooff + (long long)k * a.out.stride] = mkc(v.x * sc, v.y * (a.cj_out ? -sc : sc));
  }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    const C *in = (const C *)a.in.ptr;
    const int n = (int)a.ia;
    tile_loop(a.in, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      C *d = &line_view<C>(a, l, sb)[j];
      if (j < n) cp_async_n<sizeof(C)>(d, &in[off]);
      else *d = mkc((Rl)0, (Rl)0);
    });
  }
  // a[j] = conj?(x[j]) * w[j] for j < n
  template <class P> static GF_DEV void prep(const KArgs &a, long long, void *sb = nullptr) {
    using C = Cx<P>;
    using SP = typename P::sp_t;
    const SP *w = (const SP *)a.aux0;
    const int n = (int)a.ia;
    smem_loop(a, n, [&](int l, int j) {
      const LineView<C> s = line_view<C>(a, l, sb);
      C v = s[j];
      if (a.cj_in) v.y = -v.y;
      s[j] = spmul(v, __ldg(&w[j]));
    });
    __syncthreads();
  }
  template <class P> static GF_DEV void mid(const KArgs &a, long long, bool, void *sb = nullptr) {
    using C = Cx<P>;
    using SP = typename P::sp_t;
    const SP *B = (const SP *)a.aux2;
    smem_loop(a, a.lp.n, [&](int l, int k) {
      const LineView<C> s = line_view<C>(a, l, sb);
      s[k] = cconj(spmul(s[k], __ldg(&B[k])));
    });
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    using SP = typename P::sp_t;
    C *out = (C *)a.out.ptr;
    const SP *w = (const SP *)a.aux0;
    const int n = (int)a.ia;
    const Rl sc = (Rl)a.scale;
    const Rl sy = a.cj_out ? -sc : sc;
    tile_loop(a.out, a.lpc, n, FastDiv((uint32_t)n), a.lpcdiv, line0, a.nlines,
              [&](int l, int k, long long off) {
                C y = spmul(cconj(line_view<C>(a, l, sb)[k]), __ldg(&w[k]));
                out[off] = mkc(y.x * sc, y.y * sy);
              });
  }
};

// ---------------------------------------------------------------------------
// Spectrogram frame (freq.go:107-127 with PSD freq.go:69-90): line t is the
// frame x[t*step .. t*step+seg) times the window, transformed as an even
// real line (seg = 2m) and reduced to the one-sided density
//   p[k] = |X[k]|^2 * scale, doubled except for k = 0 and k = m.
// in: real signal (Side: dist_b = step per frame, stride 1); aux1 = window
// (real, seg); aux0 = W_2m^k table (FP32-mixed: aux2 = its FP32 hi parts,
// for short lines); out: real bins (m+1 per frame).
// ---------------------------------------------------------------------------
struct OpSpectro {
  static constexpr bool kConv = false, kFG = true, kTG = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &a, const LineCtx &c, int j) {
    using Rl = typename P::real;
    if (!c.valid) return mkc((Rl)0, (Rl)0);
    const Rl *win = (const Rl *)a.aux1;
    // direct first stage only for pair-aligned frames: pair j is one vector
    const Cx<P> v = ld_stream(reinterpret_cast<const Cx<P> *>((const Rl *)a.in.ptr + c.ioff) + j);
    return mkc(v.x * ld_keep(&win[2 * j]), v.y * ld_keep(&win[2 * j + 1]));
  }
  template <class P> static GF_DEV void gstore(const KArgs &, const LineCtx &, int, Cx<P>) {}
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    tile_loop(a.in, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      // stride 1: complex element j sits at off = line + j; its real pair is
      // at line + 2j = off + j
      load_real_pair<P>(a, &line_view<Cx<P>>(a, l, sb)[j], off + j, 1);
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &a, long long, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    const Rl *win = (const Rl *)a.aux1;
    const int m = a.lp.n;
    smem_loop(a, m, [&](int l, int j) {
      const LineView<C> s = line_view<C>(a, l, sb);
      C v = s[j];
      s[j] = mkc(v.x * __ldg(&win[2 * j]), v.y * __ldg(&win[2 * j + 1]));
    });
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using Rl = typename P::real;
    Rl *out = (Rl *)a.out.ptr;
    const Rl sc = (Rl)a.scale;
    const int m = a.lp.n;
    untangle_tile<P>(a, line0, [&](long long base, int k, Cx<P> v) {
      Rl pw = (v.x * v.x + v.y * v.y) * sc;
      if (k != 0 && k != m) pw *= (Rl)2;
      out[base + k] = pw;
    }, sb);
  }
  // Row-layout fast paths for the compiled-schedule kernels (M = lp.n).
  static constexpr bool kRowFast = true;
  template <class P, int M, int T> static GF_DEV void load_row(const KArgs &a, const LineCtx &, long long line0) {
    load<P>(a, line0);
  }
  template <class P, int M, int T> static GF_DEV void prep_row(const KArgs &a, const LineCtx &, Cx<P> *) {
    prep<P>(a, 0);
  }
  template <class P, int M, int T> static GF_DEV void store_row(const KArgs &a, const LineCtx &c, Cx<P> *sb) {
    using C = Cx<P>;
    using Rl = typename P::real;
    using TW = typename P::tw_t;
    if (!c.valid) return;
    constexpr int H = M / 2 + 1;
    constexpr int IT = (H + T - 1) / T;
    const TW *tw = (const TW *)a.aux0;
    Rl *out = (Rl *)a.out.ptr + c.ooff;
    const Rl half = (Rl)0.5;
    const Rl sc = (Rl)a.scale, sc2 = (Rl)2 * (Rl)a.scale;
#pragma unroll
    for (int it = 0; it < IT; it++) {
      const int k = c.t + it * T;
      if (IT * T > H && k >= H) break;
      if (k == 0) {
        const C z0 = sb[0];
        const Rl d0 = z0.x + z0.y, dm = z0.x - z0.y;
        out[0] = d0 * d0 * sc;
        out[M] = dm * dm * sc;
        continue;
      }
      const C zk = sb[spad(k)], zm = sb[spad(M - k)];
      const C xe = mkc((zk.x + zm.x) * half, (zk.y - zm.y) * half);
      const C xo = mkc((zk.y + zm.y) * half, (zm.x - zk.x) * half);
      C t;
      if constexpr (short_tw<P, M>()) t = cmul(xo, ld_keep(&((const float2 *)a.aux2)[k]));
      else t = twmul(xo, ld_keep(&tw[k]));
      const C lo = cadd(xe, t), hi = mkc(xe.x - t.x, t.y - xe.y);
      out[k] = (lo.x * lo.x + lo.y * lo.y) * sc2;
      if (M - k != k) out[M - k] = (hi.x * hi.x + hi.y * hi.y) * sc2;
    }
  }
};


// ---------------------------------------------------------------------------
// Rader through a two-pass (four-step) convolution, for primes whose
// convolution length cl = N1 * N2 does not fit one CTA.  Four line-kernel
// phases per signal, all on the shared-memory prologue/epilogue:
//   FS1  columns n2 of the conv signal a[n2 + N2 n1] = x[perm[..]] (zero past
//        q), FFT over n1, twiddle W_cl^{n2 k1}; stashes x0 per signal
//   FS2  rows k1, FFT over n2, output k = k1 + N1 k2 becomes conj(A[k] B[k]);
//        records X[0] = x0 + A[0] per signal
//   FS3  the plain twiddled column pass (OpC2CTwiddle) of the second FFT
//   FS4  rows, FFT, and the scatter X[iperm[k - off]] = x0 + conj(v) for
//        off <= k < off + q, plus X[0]
// Signals of the phase are batches b; lines within a signal are the
// sides' lpb groups.
// ---------------------------------------------------------------------------
struct OpRaderFS1 {  // aux0 perm, aux1 split W_cl table (2^ic + ...), aux2 x0s; ia = cl, ib = q
  static constexpr bool kConv = false, kFG = false, kTG = false;
  static GF_DEV bool first_conj(const KArgs &a) { return a.cj_in; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &, const LineCtx &, int) { return Cx<P>(); }
  template <class P> static GF_DEV void gstore(const KArgs &, const LineCtx &, int, Cx<P>) {}
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    const C *in = (const C *)a.in.ptr;
    const int *perm = (const int *)a.aux0;
    const int q = (int)a.ib;
    const int N2 = (int)a.in.lpb.d;
    const int n1len = a.lp.n;
    const int total = a.lpc * n1len;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = e / n1len, i = e - l * n1len;
      const long long gl = line0 + l;
      if (gl >= a.nlines) continue;
      uint32_t b, n2;
      a.in.lpb.divmod((uint32_t)gl, b, n2);
      const long long base = line_off(a.in, (uint32_t)gl);  // signal base (dist_l = 0)
      const int n = (int)n2 + N2 * i;
      C *d = &line_view<C>(a, l, sb)[i];
      if (n < q) cp_async_n<sizeof(C)>(d, &in[base + (long long)__ldg(&perm[n]) * a.in.stride]);
      else *d = mkc((Rl)0, (Rl)0);
      if (n == 0) {
        C x0 = in[base];
        if (a.cj_in) x0.y = -x0.y;
        ((C *)a.aux2)[b] = x0;
      }
    }
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using TW = typename P::tw_t;
    C *out = (C *)a.out.ptr;
    tile_loop(a.out, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int i, long long off) {
      uint32_t b, n2;
      a.out.lpb.divmod((uint32_t)(line0 + l), b, n2);
      // n2 < N2, i < N1: the exponent is below cl, no reduction
      out[off] = split_tw<P>(line_view<C>(a, l, sb)[i], (const TW *)a.aux1, n2 * (uint32_t)i, a.ic);
    });
  }
};

struct OpRaderFS2 {  // aux0 B/cl spectrum, aux1 x0s, aux2 dc
  static constexpr bool kConv = false, kFG = false, kTG = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &, const LineCtx &, int) { return Cx<P>(); }
  template <class P> static GF_DEV void gstore(const KArgs &, const LineCtx &, int, Cx<P>) {}
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    OpC2C::load<P>(a, line0, sb);
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using SP = typename P::sp_t;
    C *out = (C *)a.out.ptr;
    const int N1 = (int)a.out.lpb.d;
    tile_loop(a.out, a.lpc, a.lp.n, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int k2, long long off) {
      uint32_t b, k1;
      a.out.lpb.divmod((uint32_t)(line0 + l), b, k1);
      const long long k = (long long)k1 + (long long)N1 * k2;
      const C v = line_view<C>(a, l, sb)[k2];
      if (k == 0) ((C *)a.aux2)[b] = cadd(((const C *)a.aux1)[b], v);
      out[off] = cconj(spmul(v, __ldg(&((const SP *)a.aux0)[k])));
    });
  }
};

struct OpRaderFS4 {  // aux0 iperm, aux1 x0s, aux2 dc; ia = q, ib = off
  static constexpr bool kConv = false, kFG = false, kTG = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV Cx<P> gload(const KArgs &, const LineCtx &, int) { return Cx<P>(); }
  template <class P> static GF_DEV void gstore(const KArgs &, const LineCtx &, int, Cx<P>) {}
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    OpC2C::load<P>(a, line0, sb);
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    C *out = (C *)a.out.ptr;
    const int N1 = (int)a.out.lpb.d;
    const int q = (int)a.ia;
    const int offc = (int)a.ib;
    const Rl sc = (Rl)a.scale;
    const Rl sy = a.cj_out ? -sc : sc;
    const int n2len = a.lp.n;
    const int total = a.lpc * n2len;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = e / n2len, k2 = e - l * n2len;
      const long long gl = line0 + l;
      if (gl >= a.nlines) continue;
      uint32_t b, k1;
      a.out.lpb.divmod((uint32_t)gl, b, k1);
      const long long base = line_off(a.out, (uint32_t)gl);  // signal base (dist_l = 0)
      const long long k = (long long)k1 + (long long)N1 * k2;
      if (k == 0) {
        const C d = ((const C *)a.aux2)[b];
        out[base] = mkc(d.x * sc, d.y * sy);
      }
      const long long qi = k - offc;
      if (qi < 0 || qi >= q) continue;
      const C y = cadd(((const C *)a.aux1)[b], cconj(line_view<C>(a, l, sb)[k2]));
      out[base + (long long)__ldg(&((const int *)a.aux0)[qi]) * a.out.stride] = mkc(y.x * sc, y.y * sy);
    }
  }
};


// ---------------------------------------------------------------------------
// 2-D spectral filter, column part: for column k of an image's row-transformed
// spectrum (length R = lp.n, lines = (image b, column k), column-mode sides),
//   X = FFT_R(column)            (saved to aux1 when GF_FILT_SAVE)
//   G = X                        (when GF_FILT_DH: dH partial of image b,
//                                 conj(Xsaved) * w_k * da  -> aux2)
//   Y = X * H[:, k]              (conj(H) with GF_FILT_CONJ)
//   out = IFFT_R(Y) * scale      as conj(FFT(conj Y)) / ...
// H is aux0 (R x K row-major, the data's complex type); ia = C (real row
// length, for the edge-bin weight w_k = 1 at k = 0 and k = C/2, else 2).
// This fuses the forward column FFT of RFFT2, the filter multiply and the
// column IFFT of IRFFT2 (and, for the adjoint, the dH accumulation).
// ---------------------------------------------------------------------------
#define GF_FILT_CONJ 1
#define GF_FILT_SAVE 2
#define GF_FILT_DH 4

struct OpFilterCol {
  static constexpr bool kConv = true, kFG = true, kTG = true;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  // direct first stage of the forward FFT and last stage of the inverse
  template <class P> static GF_DEV Cx<P> gload(const KArgs &a, const LineCtx &c, int i) {
    return OpC2C::gload<P>(a, c, i);
  }
  template <class P> static GF_DEV void gstore(const KArgs &a, const LineCtx &c, int i, Cx<P> y) {
    OpC2C::gstore<P>(a, c, i, y);
  }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0, void *sb = nullptr) {
    OpC2C::load<P>(a, line0, sb);
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long, void * = nullptr) {}
  template <class P> static GF_DEV void mid(const KArgs &a, long long line0, bool, void *sb = nullptr) {
    using C = Cx<P>;
    using Rl = typename P::real;
    const C *H = (const C *)a.aux0;
    C *xs = (C *)a.aux1;
    C *dh = (C *)a.aux2;
    const int R = a.lp.n;
    const int K = (int)a.out.lpb.d;
    const int Cn = (int)a.ia;
    tile_loop(a.out, a.lpc, R, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int r, long long off) {
      uint32_t b, k;
      a.out.lpb.divmod((uint32_t)(line0 + l), b, k);
      const LineView<C> s = line_view<C>(a, l, sb);
      const C x = s[r];
      const long long hi = (long long)r * K + k;            // H index
      const long long pi = (long long)b * R * K + hi;       // per-image spectrum index
      if (a.ic & GF_FILT_SAVE) xs[pi] = x;
      if (a.ic & GF_FILT_DH) {
        const Rl w = (k == 0 || 2 * (int)k == Cn) ? (Rl)1 : (Rl)2;
        const C xb = xs[pi];
        const Rl sc = w * (Rl)a.da;
        // conj(Xsaved) * G * w / (R C)
        dh[pi] = mkc((xb.x * x.x + xb.y * x.y) * sc, (xb.x * x.y - xb.y * x.x) * sc);
      }
      C h = H[hi];
      if (a.ic & GF_FILT_CONJ) h.y = -h.y;
      s[r] = cconj(cmul(x, h));
      (void)off;
    });
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0, void *sb = nullptr) {
    OpC2C::store<P>(a, line0, sb);  // conj and 1/R via cj_out and scale
  }
};

}  // namespace gf
