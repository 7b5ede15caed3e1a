// kernels.cuh -- fused convolution ops (Rader, Bluestein), the spectrogram
// op, the line kernel itself, and the elementwise kernels used by multi-pass
// plans and plan construction (twiddle, chirp and permutation tables).
#pragma once
#include <type_traits>
#include "engine.cuh"

namespace gf {

// ---------------------------------------------------------------------------
// Rader, fused in one CTA (rader.go:129-172 restated for one line):
//   a[k] = x[perm[k]] (k < q = p-1, zero-padded to cl), A = FFT_cl(a),
//   X[0] = x0 + A[0] (= sum of all inputs),
//   conv = IFFT_cl(A * B)  evaluated as conj(FFT_cl(conj(A * B / cl))),
//   X[iperm[qi]] = x0 + conv[qi + off]   (off = 0 cyclic, q padded-linear).
// aux0 = perm (int32, q), aux1 = iperm (int32, q), aux2 = B/cl (sp_t, cl),
// ia = p, ic = off.  lp is the length-cl program.
// ---------------------------------------------------------------------------
struct OpRader {
  static constexpr bool kConv = true;
  static GF_DEV bool first_conj(const KArgs &a) { return a.cj_in; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    const C *in = (const C *)a.in.ptr;
    const int *perm = (const int *)a.aux0;
    const int cl = a.lp.n;
    const int q = (int)a.ia - 1;
    const bool cj = a.cj_in;
    const long long st = a.in.stride;
    tile_loop(a.in, a.lpc, cl, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int k, long long off) {
      const long long base = off - (long long)k * st;
      C *d = &line_buf<P>(l, cl)[spad(k)];
      if (k < q) cp_async_n<sizeof(C)>(d, &in[base + (long long)__ldg(&perm[k]) * st]);
      else *d = mkc((Rl)0, (Rl)0);
      if (k == 0) {
        C x0 = in[base];
        if (cj) x0.y = -x0.y;
        line_extra<P>(l, cl, a.lpc)[0] = x0;
      }
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &, long long) {}
  template <class P> static GF_DEV void mid(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using SP = typename P::sp_t;
    const SP *B = (const SP *)a.aux2;
    const int cl = a.lp.n;
    // DC first (reads A[0] before the multiply overwrites it)
    for (int l = threadIdx.x; l < a.lpc; l += blockDim.x) {
      C *ex = line_extra<P>(l, cl, a.lpc);
      ex[1] = cadd(ex[0], line_buf<P>(l, cl)[spad(0)]);
    }
    __syncthreads();
    const int total = a.lpc * cl;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      uint32_t l, k;
      a.ndiv.divmod((uint32_t)e, l, k);
      C *s = line_buf<P>((int)l, cl);
      s[spad(k)] = cconj(spmul(s[spad(k)], __ldg(&B[k])));
    }
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    C *out = (C *)a.out.ptr;
    const int *iperm = (const int *)a.aux1;
    const int cl = a.lp.n;
    const int p = (int)a.ia;
    const int q = p - 1;
    const int offc = a.ic;
    const Rl sc = (Rl)a.scale;
    const Rl sy = a.cj_out ? -sc : sc;
    const long long st = a.out.stride;
    tile_loop(a.out, a.lpc, p, FastDiv((uint32_t)p), a.lpcdiv, line0, a.nlines,
              [&](int l, int i, long long off) {
                const long long base = off - (long long)i * st;
                const C *ex = line_extra<P>(l, cl, a.lpc);
                C y;
                long long dst;
                if (i == 0) {
                  y = ex[1];
                  dst = 0;
                } else {
                  const int qi = i - 1;
                  C c = cconj(line_buf<P>(l, cl)[spad(qi + offc)]);
                  y = cadd(ex[0], c);
                  dst = __ldg(&iperm[qi]);
                }
                (void)q;
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
  static constexpr bool kConv = true;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    const C *in = (const C *)a.in.ptr;
    const int m = a.lp.n;
    const int n = (int)a.ia;
    tile_loop(a.in, a.lpc, m, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      C *d = &line_buf<P>(l, m)[spad(j)];
      if (j < n) cp_async_n<sizeof(C)>(d, &in[off]);
      else *d = mkc((Rl)0, (Rl)0);
    });
  }
  // a[j] = conj?(x[j]) * w[j] for j < n
  template <class P> static GF_DEV void prep(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using SP = typename P::sp_t;
    const SP *w = (const SP *)a.aux0;
    const int m = a.lp.n;
    const int n = (int)a.ia;
    const bool cj = a.cj_in;
    for (int e = threadIdx.x; e < a.lpc * n; e += blockDim.x) {
      const int l = e / n, j = e - l * n;
      C *s = line_buf<P>(l, m);
      C v = s[spad(j)];
      if (cj) v.y = -v.y;
      s[spad(j)] = spmul(v, __ldg(&w[j]));
    }
    __syncthreads();
    (void)line0;
  }
  template <class P> static GF_DEV void mid(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using SP = typename P::sp_t;
    const SP *B = (const SP *)a.aux2;
    const int m = a.lp.n;
    const int total = a.lpc * m;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      uint32_t l, k;
      a.ndiv.divmod((uint32_t)e, l, k);
      C *s = line_buf<P>((int)l, m);
      s[spad(k)] = cconj(spmul(s[spad(k)], __ldg(&B[k])));
    }
    __syncthreads();
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    using SP = typename P::sp_t;
    C *out = (C *)a.out.ptr;
    const SP *w = (const SP *)a.aux0;
    const int m = a.lp.n;
    const int n = (int)a.ia;
    const Rl sc = (Rl)a.scale;
    const Rl sy = a.cj_out ? -sc : sc;
    tile_loop(a.out, a.lpc, n, FastDiv((uint32_t)n), a.lpcdiv, line0, a.nlines,
              [&](int l, int k, long long off) {
                C y = spmul(cconj(line_buf<P>(l, m)[spad(k)]), __ldg(&w[k]));
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
// (real, seg); aux0 = W_2m^k table; out: real bins (m+1 per frame).
// ---------------------------------------------------------------------------
struct OpSpectro {
  static constexpr bool kConv = false;
  static GF_DEV bool first_conj(const KArgs &) { return false; }
  template <class P> static GF_DEV void load(const KArgs &a, long long line0) {
    const int m = a.lp.n;
    tile_loop(a.in, a.lpc, m, a.ndiv, a.lpcdiv, line0, a.nlines, [&](int l, int j, long long off) {
      // stride 1: complex element j sits at off = line + j; its real pair is
      // at line + 2j = off + j
      load_real_pair<P>(a, &line_buf<P>(l, m)[spad(j)], off + j, 1);
    });
  }
  template <class P> static GF_DEV void prep(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    const Rl *win = (const Rl *)a.aux1;
    const int m = a.lp.n;
    for (int e = threadIdx.x; e < a.lpc * m; e += blockDim.x) {
      const int l = e / m, j = e - l * m;
      C *s = line_buf<P>(l, m);
      C v = s[spad(j)];
      s[spad(j)] = mkc(v.x * __ldg(&win[2 * j]), v.y * __ldg(&win[2 * j + 1]));
    }
    __syncthreads();
    (void)line0;
  }
  template <class P> static GF_DEV void store(const KArgs &a, long long line0) {
    using C = typename P::cpx;
    using Rl = typename P::real;
    using TW = typename P::tw_t;
    Rl *out = (Rl *)a.out.ptr;
    const TW *tw = (const TW *)a.aux0;
    const int m = a.lp.n;
    const int h = m / 2 + 1;
    const Rl half = (Rl)0.5;
    const Rl sc = (Rl)a.scale;
    tile_loop(a.out, a.lpc, h, FastDiv((uint32_t)h), a.lpcdiv, line0, a.nlines,
              [&](int l, int k, long long off) {
                const C *s = line_buf<P>(l, m);
                const long long base = off - k;
                if (k == 0) {
                  C z0 = s[spad(0)];
                  const Rl d0 = z0.x + z0.y, dm = z0.x - z0.y;
                  out[base] = d0 * d0 * sc;
                  out[base + m] = dm * dm * sc;
                  return;
                }
                C zk = s[spad(k)], zm = s[spad(m - k)];
                C xe = mkc((zk.x + zm.x) * half, (zk.y - zm.y) * half);
                C xo = mkc((zk.y + zm.y) * half, (zm.x - zk.x) * half);
                C t = twmul(xo, __ldg(&tw[k]));
                C xk = cadd(xe, t);
                out[off] = (xk.x * xk.x + xk.y * xk.y) * sc * (Rl)2;
                if (m - k != k) {
                  C xm = csub(xe, t);
                  out[base + (m - k)] = (xm.x * xm.x + xm.y * xm.y) * sc * (Rl)2;
                }
              });
  }
};

// ---------------------------------------------------------------------------
// The line kernel: prologue, stages, [spectrum multiply, stages], epilogue.
// ---------------------------------------------------------------------------
template <class P, int MAXE, class Op>
__global__ void __launch_bounds__(512, 1) k_line(const KArgs a) {
  const long long line0 = (long long)blockIdx.x * a.lpc;
  Op::template load<P>(a, line0);
  cp_async_wait_all();
  __syncthreads();
  Op::template prep<P>(a, line0);
  const int l = threadIdx.x / a.lp.T;
  const int t = threadIdx.x - l * a.lp.T;
  typename P::cpx *s = line_buf<P>(l, a.lp.n);
  run_stages<P, MAXE>(s, a.lp, t, Op::first_conj(a));
  if constexpr (Op::kConv) {
    Op::template mid<P>(a, line0);
    run_stages<P, MAXE>(s, a.lp, t, false);
  }
  Op::template store<P>(a, line0);
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

// W_L^k for k = 0..count-1 (four-step and real-untangle tables).
template <class TW> __global__ void k_gen_roots(TW *tw, long long L, long long count) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x)
    put_tw(tw, k, root_of_unity(k, L));
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
__global__ void k_untangle(Side dst, const C *Z, long long nlines, int m, const TW *tw) {
  using Rl = decltype(C().x);
  const int h = m / 2 + 1;
  const long long total = nlines * h;
  const Rl half = (Rl)0.5;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / h;
    const int k = (int)(e - l * h);
    const C *z = Z + l * m;
    C *o = (C *)dst.ptr + line_off(dst, (uint32_t)l);
    const long long st = dst.stride;
    if (k == 0) {
      C z0 = z[0];
      o[0] = mkc(z0.x + z0.y, (Rl)0);
      o[(long long)m * st] = mkc(z0.x - z0.y, (Rl)0);
      continue;
    }
    C zk = z[k], zm = z[m - k];
    C xe = mkc((zk.x + zm.x) * half, (zk.y - zm.y) * half);
    C xo = mkc((zk.y + zm.y) * half, (zm.x - zk.x) * half);
    C t = twmul(xo, tw[k]);
    o[(long long)k * st] = cadd(xe, t);
    if (m - k != k) o[(long long)(m - k) * st] = mkc(xe.x - t.x, t.y - xe.y);
  }
}

GF_DEV double2 conj_tw(double2 w) { return make_double2(w.x, -w.y); }
GF_DEV float2 conj_tw(float2 w) { return make_float2(w.x, -w.y); }
GF_DEV float4 conj_tw(float4 w) { return make_float4(w.x, -w.y, w.z, -w.w); }

// Reverse untangle (realplan.go:235-272) from bins of `src` (nb per line
// available) into conjugated packed spectra Z (m per line, contiguous).
template <class C, class TW>
__global__ void k_reverse_untangle(C *Z, Side src, long long nlines, int m, int nb, const TW *tw) {
  using Rl = decltype(C().x);
  const int h = m / 2 + 1;
  const long long total = nlines * h;
  const Rl half = (Rl)0.5;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / h;
    const int k = (int)(e - l * h);
    const C *in = (const C *)src.ptr + line_off(src, (uint32_t)l);
    const long long st = src.stride;
    auto bin = [&](int q) -> C { return q < nb ? in[(long long)q * st] : mkc((Rl)0, (Rl)0); };
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
__global__ void k_copy_bins(Side dst, const C *src, long long nlines, int n) {
  const int h = n / 2 + 1;
  const long long total = nlines * h;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / h;
    const int k = (int)(e - l * h);
    ((C *)dst.ptr)[line_off(dst, (uint32_t)l) + (long long)k * dst.stride] = src[l * n + k];
  }
}

// Hermitian mirror (realplan.go:197-206) of bins (nb available) into
// conjugated full lines of length n, contiguous.
template <class C>
__global__ void k_mirror(C *dst, Side src, long long nlines, int n, int nb) {
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
