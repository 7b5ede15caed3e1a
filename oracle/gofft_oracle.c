/*
 * gofft_oracle.c -- CPU restatement of go-fft/fft's transform path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine and the timed CPU
 * baseline.  The product path never links or calls this file.
 *
 * Compile with -O2 -ffp-contract=off (no -ffast-math): Go on amd64 never fuses
 * multiply-add, and the reference's bit-identity tests depend on that
 * (internal/kernels/butterfly.go:29-37, cmul.go:16-24).  Each function cites
 * the reference file:line it restates.
 */
#define _GNU_SOURCE
#include "gofft_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef struct { double re, im; } cx;

static inline cx mk(double re, double im) { cx z; z.re = re; z.im = im; return z; }
static inline cx cadd(cx a, cx b) { return mk(a.re + b.re, a.im + b.im); }
static inline cx csub(cx a, cx b) { return mk(a.re - b.re, a.im - b.im); }
/* Go's complex128 product: (ar*br - ai*bi) + (ar*bi + ai*br)i, separately
 * rounded (internal/kernels/butterfly.go:123-127, cmul.go:26-36). */
static inline cx cmul(cx a, cx b) {
  return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline cx cconj(cx a) { return mk(a.re, -a.im); }

static void *xmalloc(size_t n) {
  void *p = malloc(n ? n : 1);
  if (!p) abort();
  return p;
}
static cx *cxalloc(size_t n) { return (cx *)calloc(n ? n : 1, sizeof(cx)); }

/* ======================================================================== */
/* Integer helpers                                                          */
/* ======================================================================== */

/* plan.go:134-141 */
int or_factors_small(int n) {
  static const int primes[6] = {2, 3, 5, 7, 11, 13};
  for (int i = 0; i < 6; i++)
    while (n % primes[i] == 0) n /= primes[i];
  return n == 1;
}

/* plan.go:265-279: 4s first, then ascending small primes. */
int or_factorize(int n, int *out) {
  int c = 0;
  while (n % 4 == 0) { out[c++] = 4; n /= 4; }
  static const int primes[6] = {2, 3, 5, 7, 11, 13};
  for (int i = 0; i < 6; i++)
    while (n % primes[i] == 0) { out[c++] = primes[i]; n /= primes[i]; }
  return c;
}

/* plan.go:154-173 */
int or_next_smooth_conv(int lo) {
  if (lo < 1) lo = 1;
  for (int m = lo;; m++) {
    int x = m;
    while (x % 2 == 0) x /= 2;
    while (x % 3 == 0) x /= 3;
    while (x % 5 == 0) x /= 5;
    if (x == 1) return m;
  }
}

/* plan.go:192-220 */
int or_conv_cost(int m, double *cost_out) {
  const double w2 = 2.0, w3 = 2.0, w5 = 2.8, w7 = 2.6;
  double cost = 0.0;
  int x = m;
  while (x % 4 == 0) { cost += w2; x /= 4; }
  while (x % 2 == 0) { cost += w2; x /= 2; }
  while (x % 3 == 0) { cost += w3; x /= 3; }
  while (x % 5 == 0) { cost += w5; x /= 5; }
  while (x % 7 == 0) { cost += w7; x /= 7; }
  if (x != 1) { if (cost_out) *cost_out = 0; return 0; }
  if (cost_out) *cost_out = (double)m * cost;
  return 1;
}

/* plan.go:241-259: argmin of convCost over [lo, lo + ceil(0.4 lo)]. */
int or_best_conv_len(int lo) {
  if (lo < 1) lo = 1;
  int hi = lo + (lo * 4 + 9) / 10;
  int best = lo;
  double best_cost = 0;
  or_conv_cost(lo, &best_cost);
  int have = 0;
  for (int m = lo; m <= hi; m++) {
    double c;
    if (!or_conv_cost(m, &c)) continue;
    if (!have || c < best_cost) { best = m; best_cost = c; have = 1; }
  }
  return best;
}

/* rader.go:232-245 */
int or_is_prime(int n) {
  if (n < 2) return 0;
  if (n % 2 == 0) return n == 2;
  for (int d = 3; d * d <= n; d += 2)
    if (n % d == 0) return 0;
  return 1;
}

/* rader.go:217-228 */
static int64_t mod_pow(int64_t base, int64_t e, int64_t m) {
  int64_t r = 1;
  base %= m;
  while (e > 0) {
    if (e & 1) r = r * base % m;
    e >>= 1;
    base = base * base % m;
  }
  return r;
}

/* rader.go:178-212 */
int or_primitive_root(int p) {
  int phi = p - 1;
  int f[32], nf = 0, m = phi;
  for (int d = 2; d * d <= m; d++) {
    if (m % d == 0) {
      f[nf++] = d;
      while (m % d == 0) m /= d;
    }
  }
  if (m > 1) f[nf++] = m;
  if (nf == 0) return 1;
  for (int g = 2;; g++) {
    int gen = 1;
    for (int i = 0; i < nf; i++)
      if (mod_pow(g, phi / f[i], p) == 1) { gen = 0; break; }
    if (gen) return g;
  }
}

/* plan.go:42-73 routing. */
#define RADER_THRESHOLD 700
int or_engine(int n) {
  if (n <= 1) return OR_TRIVIAL;
  if ((n & (n - 1)) == 0) return OR_IT;
  if (or_factors_small(n)) return OR_CT;
  if (n >= RADER_THRESHOLD && or_is_prime(n)) return OR_RADER;
  return OR_BLUESTEIN;
}

/* iterative.go:59-80: a leading radix-2 when log2 n is odd, then radix-4s. */
int or_it_radices(int n, int *out) {
  int lg = 0;
  while ((1 << lg) < n) lg++;
  int c = 0;
  if (lg % 2 == 1) out[c++] = 2;
  for (int i = 0; i < lg / 2; i++) out[c++] = 4;
  return c;
}

/* iterative.go:87-103: mixed-radix digit reversal. */
static void rev_for_radices(int n, const int *rad, int nr, int *rev) {
  for (int i = 0; i < n; i++) {
    int x = i, r = 0;
    for (int s = 0; s < nr; s++) {
      r = r * rad[s] + x % rad[s];
      x /= rad[s];
    }
    rev[i] = r;
  }
}

void or_rev_pos(int n, int *out) {
  int rad[64];
  int nr = or_it_radices(n, rad);
  rev_for_radices(n, rad, nr, out);
}

/* kernels.go:20-32, expressed as the permutation it applies:
 * after BitReverse, x'[i] = x[out[i]]. */
void or_bit_reverse_perm(int n, int *out) {
  for (int i = 0; i < n; i++) out[i] = i;
  for (int i = 1, j = 0; i < n; i++) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) { int t = out[i]; out[i] = out[j]; out[j] = t; }
  }
}

/* ======================================================================== */
/* Plans                                                                    */
/* ======================================================================== */

/* plan.go:320-327: exp(-2 pi i k / n) via cos/sin of the same expression. */
static cx *twiddle_table(int n) {
  cx *t = cxalloc(n);
  for (int k = 0; k < n; k++) {
    double ang = -2 * M_PI * (double)k / (double)n;
    t[k] = mk(cos(ang), sin(ang));
  }
  return t;
}

typedef struct { int radix, span; cx *tw, *twc; } it_stage;
typedef struct { int n, nst; int *rev; it_stage st[40]; } it_plan;
typedef struct { int n, nf; int f[64]; cx *tw, *twc; } ct_plan;
typedef struct { int n, cl, cyclic; int *perm, *iperm; cx *bF, *bI; } rader_plan;
typedef struct { int n, m; cx *wF, *wI, *bF, *bI; } blue_plan;
typedef struct {
  int n;
  it_plan *it;
  ct_plan *ct;
  rader_plan *rader;
  blue_plan *blue;
} or_plan;

static or_plan *cached_plan(int n);
static void plan_fft(or_plan *p, cx *dst, const cx *src);
static void plan_ifft(or_plan *p, cx *dst, const cx *src);
static void plan_execute(or_plan *p, cx *dst, const cx *src, int inverse);

/* iterative.go:59-150 */
static it_plan *new_it_plan(int n) {
  it_plan *p = (it_plan *)calloc(1, sizeof(it_plan));
  p->n = n;
  int rad[40];
  int nr = or_it_radices(n, rad);
  p->rev = (int *)xmalloc(sizeof(int) * n);
  rev_for_radices(n, rad, nr, p->rev);
  cx *root = twiddle_table(n);
  int span = 1;
  p->nst = nr;
  for (int s = 0; s < nr; s++) {
    int r = rad[s], next = span * r;
    it_stage *st = &p->st[s];
    st->radix = r;
    st->span = span;
    if (r == 2) {
      st->tw = cxalloc(span);
      st->twc = cxalloc(span);
      for (int k = 0; k < span; k++) {
        cx w = root[((int64_t)k * (n / next)) % n];
        st->tw[k] = w;
        st->twc[k] = cconj(w);
      }
    } else {
      st->tw = cxalloc((size_t)span * 3);
      st->twc = cxalloc((size_t)span * 3);
      int step = n / next;
      for (int k = 0; k < span; k++) {
        cx w1 = root[((int64_t)k * step) % n];
        cx w2 = root[((int64_t)2 * k * step) % n];
        cx w3 = root[((int64_t)3 * k * step) % n];
        st->tw[k] = w1;
        st->tw[span + k] = w2;
        st->tw[2 * span + k] = w3;
        st->twc[k] = cconj(w1);
        st->twc[span + k] = cconj(w2);
        st->twc[2 * span + k] = cconj(w3);
      }
    }
    span = next;
  }
  free(root);
  return p;
}

/* internal/kernels/butterfly.go:53-67 */
static void radix2_stage(cx *a, int n, int span, const cx *tw) {
  if (span == 0 || n == 0) return;
  int step = 2 * span;
  for (int base = 0; base < n; base += step)
    for (int k = 0; k < span; k++) {
      int i = base + k, j = i + span;
      double hr = a[j].re, hi = a[j].im, wr = tw[k].re, wi = tw[k].im;
      cx t = mk(hr * wr - hi * wi, hr * wi + hi * wr);
      cx u = a[i];
      a[i] = cadd(u, t);
      a[j] = csub(u, t);
    }
}

/* internal/kernels/butterfly.go:80-108 */
static void radix4_stage(cx *a, int n, int span, const cx *w1, const cx *w2, const cx *w3,
                         int inverse) {
  if (span == 0 || n == 0) return;
  int step = 4 * span;
  for (int base = 0; base < n; base += step) {
    int i0 = base, i1 = i0 + span, i2 = i1 + span, i3 = i2 + span;
    for (int k = 0; k < span; k++) {
      cx m1 = cmul(a[i1 + k], w1[k]);
      cx m2 = cmul(a[i2 + k], w2[k]);
      cx m3 = cmul(a[i3 + k], w3[k]);
      cx a0 = a[i0 + k];
      cx t0 = cadd(a0, m2), t1 = csub(a0, m2), t2 = cadd(m1, m3), d = csub(m1, m3);
      cx t3 = inverse ? mk(-d.im, d.re) : mk(d.im, -d.re);
      a[i0 + k] = cadd(t0, t2);
      a[i1 + k] = cadd(t1, t3);
      a[i2 + k] = csub(t0, t2);
      a[i3 + k] = csub(t1, t3);
    }
  }
}

/* iterative.go:200-214 */
static void it_run(it_plan *p, cx *a, int inverse) {
  for (int s = 0; s < p->nst; s++) {
    it_stage *st = &p->st[s];
    const cx *tw = inverse ? st->twc : st->tw;
    if (st->radix == 2)
      radix2_stage(a, p->n, st->span, tw);
    else
      radix4_stage(a, p->n, st->span, tw, tw + st->span, tw + 2 * st->span, inverse);
  }
}

/* iterative.go:154-166 */
static void it_transform(it_plan *p, cx *dst, const cx *src, int inverse) {
  cx *tmp = NULL;
  if (dst == src) {
    tmp = cxalloc(p->n);
    memcpy(tmp, src, sizeof(cx) * p->n);
    src = tmp;
  }
  for (int i = 0; i < p->n; i++) dst[i] = src[p->rev[i]];
  free(tmp);
  it_run(p, dst, inverse);
}

/* iterative.go:191-197 */
static void it_transform_real_packed(it_plan *p, cx *dst, const double *src) {
  for (int i = 0; i < p->n; i++) {
    int j = p->rev[i];
    dst[i] = mk(src[2 * j], src[2 * j + 1]);
  }
  it_run(p, dst, 0);
}

/* iterative.go:177-183 */
static void it_transform_scratch(it_plan *p, cx *dst, const cx *scratch, int inverse) {
  for (int i = 0; i < p->n; i++) dst[i] = scratch[p->rev[i]];
  it_run(p, dst, inverse);
}

/* ---- mixed-radix Cooley-Tukey (mixedradix.go) --------------------------- */

/* mixedradix.go:28-40 */
static ct_plan *new_ct_plan(int n) {
  ct_plan *p = (ct_plan *)calloc(1, sizeof(ct_plan));
  p->n = n;
  p->tw = twiddle_table(n);
  p->twc = cxalloc(n);
  for (int i = 0; i < n; i++) p->twc[i] = cconj(p->tw[i]);
  p->nf = or_factorize(n, p->f);
  return p;
}

static const double SIN120 = 0.86602540378443864676372317075293618;

/* mixedradix.go:125-133 */
static void ct_radix2(cx *out, int m, int step, const cx *tw) {
  for (int k = 0; k < m; k++) {
    cx w = tw[(int64_t)k * step];
    cx a = out[k];
    cx b = cmul(out[k + m], w);
    out[k] = cadd(a, b);
    out[k + m] = csub(a, b);
  }
}

/* mixedradix.go:138-170 */
static void ct_radix4(cx *out, int m, int step, const cx *tw, int inverse) {
  for (int k = 0; k < m; k++) {
    int64_t ks = (int64_t)k * step;
    cx w1 = tw[ks], w2 = tw[2 * ks], w3 = tw[3 * ks];
    cx a = out[k];
    cx b = cmul(out[k + m], w1);
    cx c = cmul(out[k + 2 * m], w2);
    cx d = cmul(out[k + 3 * m], w3);
    cx t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = csub(b, d);
    cx t3r = inverse ? mk(-t3.im, t3.re) : mk(t3.im, -t3.re);
    out[k] = cadd(t0, t2);
    out[k + m] = cadd(t1, t3r);
    out[k + 2 * m] = csub(t0, t2);
    out[k + 3 * m] = csub(t1, t3r);
  }
}

/* mixedradix.go:178-200 */
static void ct_radix3(cx *out, int m, int step, const cx *tw, int inverse) {
  double s = inverse ? SIN120 : -SIN120;
  for (int k = 0; k < m; k++) {
    int64_t ks = (int64_t)k * step;
    cx w1 = tw[ks], w2 = tw[2 * ks];
    cx a = out[k];
    cx b = cmul(out[k + m], w1);
    cx c = cmul(out[k + 2 * m], w2);
    cx t = cadd(b, c);
    out[k] = cadd(a, t);
    cx u = csub(a, mk(t.re * 0.5, t.im * 0.5));
    cx d = csub(b, c);
    cx v = mk(-s * d.im, s * d.re);
    out[k + m] = cadd(u, v);
    out[k + 2 * m] = csub(u, v);
  }
}

static inline cx rot_i(cx z) { return mk(-z.im, z.re); }

/* mixedradix.go:205-242 */
static void ct_radix5(cx *out, int m, int step, const cx *tw, int inverse) {
  const double c1 = 0.30901699437494742410229341718281906;
  const double s1 = 0.95105651629515357211643933337938214;
  const double c2 = -0.80901699437494742410229341718281906;
  const double s2 = 0.58778525229247312916870595463907277;
  double sg = inverse ? 1.0 : -1.0;
  for (int k = 0; k < m; k++) {
    int64_t ks = (int64_t)k * step;
    cx a = out[k];
    cx b = cmul(out[k + m], tw[ks]);
    cx c = cmul(out[k + 2 * m], tw[2 * ks]);
    cx d = cmul(out[k + 3 * m], tw[3 * ks]);
    cx e = cmul(out[k + 4 * m], tw[4 * ks]);
    cx t1 = cadd(b, e), t2 = csub(b, e), t3 = cadd(c, d), t4 = csub(c, d);
    out[k] = cadd(cadd(a, t1), t3);
    cx r1 = cadd(a, mk(c1 * t1.re + c2 * t3.re, c1 * t1.im + c2 * t3.im));
    cx r2 = cadd(a, mk(c2 * t1.re + c1 * t3.re, c2 * t1.im + c1 * t3.im));
    cx i1 = rot_i(mk(sg * (s1 * t2.re + s2 * t4.re), sg * (s1 * t2.im + s2 * t4.im)));
    cx i2 = rot_i(mk(sg * (s2 * t2.re - s1 * t4.re), sg * (s2 * t2.im - s1 * t4.im)));
    out[k + m] = cadd(r1, i1);
    out[k + 4 * m] = csub(r1, i1);
    out[k + 2 * m] = cadd(r2, i2);
    out[k + 3 * m] = csub(r2, i2);
  }
}

/* mixedradix.go:251-298 */
static void ct_radix7(cx *out, int m, int step, const cx *tw, int inverse) {
  const double c1 = 0.62348980185873353052500488400423981;
  const double s1 = 0.78183148246802980870844452667405775;
  const double c2 = -0.22252093395631440428890256449679476;
  const double s2 = 0.97492791218182360701813168299393122;
  const double c3 = -0.90096886790241912623610231950744505;
  const double s3 = 0.43388373911755812047576833284835875;
  double sg = inverse ? 1.0 : -1.0;
  for (int k = 0; k < m; k++) {
    int64_t ks = (int64_t)k * step;
    cx a = out[k];
    cx b = cmul(out[k + m], tw[ks]);
    cx c = cmul(out[k + 2 * m], tw[2 * ks]);
    cx d = cmul(out[k + 3 * m], tw[3 * ks]);
    cx e = cmul(out[k + 4 * m], tw[4 * ks]);
    cx f = cmul(out[k + 5 * m], tw[5 * ks]);
    cx g = cmul(out[k + 6 * m], tw[6 * ks]);
    cx s16 = cadd(b, g), d16 = csub(b, g);
    cx s25 = cadd(c, f), d25 = csub(c, f);
    cx s34 = cadd(d, e), d34 = csub(d, e);
    out[k] = cadd(cadd(cadd(a, s16), s25), s34);
    cx r1 = cadd(a, mk(c1 * s16.re + c2 * s25.re + c3 * s34.re, c1 * s16.im + c2 * s25.im + c3 * s34.im));
    cx r2 = cadd(a, mk(c2 * s16.re + c3 * s25.re + c1 * s34.re, c2 * s16.im + c3 * s25.im + c1 * s34.im));
    cx r3 = cadd(a, mk(c3 * s16.re + c1 * s25.re + c2 * s34.re, c3 * s16.im + c1 * s25.im + c2 * s34.im));
    cx i1 = rot_i(mk(sg * (s1 * d16.re + s2 * d25.re + s3 * d34.re),
                     sg * (s1 * d16.im + s2 * d25.im + s3 * d34.im)));
    cx i2 = rot_i(mk(sg * (s2 * d16.re - s3 * d25.re - s1 * d34.re),
                     sg * (s2 * d16.im - s3 * d25.im - s1 * d34.im)));
    cx i3 = rot_i(mk(sg * (s3 * d16.re - s1 * d25.re + s2 * d34.re),
                     sg * (s3 * d16.im - s1 * d25.im + s2 * d34.im)));
    out[k + m] = cadd(r1, i1);
    out[k + 6 * m] = csub(r1, i1);
    out[k + 2 * m] = cadd(r2, i2);
    out[k + 5 * m] = csub(r2, i2);
    out[k + 3 * m] = cadd(r3, i3);
    out[k + 4 * m] = csub(r3, i3);
  }
}

/* mixedradix.go:310-335: O(r^2) general radix with a stack buffer. */
static void ct_radixP(ct_plan *p, cx *out, int r, int m, int step, const cx *tw) {
  int n = p->n;
  cx buf[16];
  int rstep = n / r;
  for (int k = 0; k < m; k++) {
    for (int i = 0; i < r; i++) buf[i] = cmul(out[k + i * m], tw[((int64_t)i * k * step) % n]);
    for (int q = 0; q < r; q++) {
      cx sum = mk(0, 0);
      for (int i = 0; i < r; i++) sum = cadd(sum, cmul(buf[i], tw[((int64_t)i * q * rstep) % n]));
      out[k + q * m] = sum;
    }
  }
}

/* mixedradix.go:103-119 */
static void ct_butterfly(ct_plan *p, cx *out, int length, int r, int m, const cx *tw, int inverse) {
  int step = p->n / length;
  switch (r) {
    case 2: ct_radix2(out, m, step, tw); break;
    case 3: ct_radix3(out, m, step, tw, inverse); break;
    case 4: ct_radix4(out, m, step, tw, inverse); break;
    case 5: ct_radix5(out, m, step, tw, inverse); break;
    case 7: ct_radix7(out, m, step, tw, inverse); break;
    default: ct_radixP(p, out, r, m, step, tw); break;
  }
}

/* mixedradix.go:69-97 */
static void ct_rec(ct_plan *p, cx *out, const cx *src, int length, int64_t stride, const int *factors,
                   const cx *tw, int inverse) {
  int r = factors[0];
  int m = length / r;
  if (m == 1) {
    for (int i = 0; i < r; i++) out[i] = src[i * stride];
  } else {
    for (int i = 0; i < r; i++)
      ct_rec(p, out + (int64_t)i * m, src + i * stride, m, r * stride, factors + 1, tw, inverse);
  }
  ct_butterfly(p, out, length, r, m, tw, inverse);
}

/* mixedradix.go:55-62 */
static void ct_transform(ct_plan *p, cx *dst, const cx *src, int inverse) {
  cx *scratch = cxalloc(p->n);
  memcpy(scratch, src, sizeof(cx) * p->n);
  ct_rec(p, dst, scratch, p->n, 1, p->f, inverse ? p->twc : p->tw, inverse);
  free(scratch);
}

/* ---- Rader (rader.go) ---------------------------------------------------- */

/* rader.go:101-125 */
static cx *rader_kernel(rader_plan *p, int n, int inverse) {
  int q = n - 1;
  cx *b = cxalloc(p->cl);
  double sign = inverse ? 1.0 : -1.0;
  int lim = p->cyclic ? q : 2 * q;
  for (int m = 0; m < lim; m++) {
    int s = m % q;
    int e = p->perm[(q - s) % q];
    double ang = sign * 2 * M_PI * (double)e / (double)n;
    b[m] = mk(cos(ang), sin(ang));
  }
  cx *out = cxalloc(p->cl);
  plan_fft(cached_plan(p->cl), out, b);
  free(b);
  return out;
}

/* rader.go:51-91 */
static rader_plan *new_rader_plan(int n) {
  int g = or_primitive_root(n);
  int q = n - 1;
  rader_plan *p = (rader_plan *)calloc(1, sizeof(rader_plan));
  p->n = n;
  if (or_factors_small(q)) {
    p->cyclic = 1;
    p->cl = q;
  } else {
    p->cl = or_best_conv_len(2 * q);
  }
  p->perm = (int *)xmalloc(sizeof(int) * q);
  p->iperm = (int *)xmalloc(sizeof(int) * q);
  int64_t x = 1;
  for (int k = 0; k < q; k++) {
    p->perm[k] = (int)x;
    x = x * g % n;
  }
  for (int qi = 0; qi < q; qi++) p->iperm[qi] = p->perm[(q - qi) % q];
  p->bF = rader_kernel(p, n, 0);
  p->bI = rader_kernel(p, n, 1);
  return p;
}

/* rader.go:129-172 */
static void rader_transform(rader_plan *p, cx *dst, const cx *src, int inverse) {
  int n = p->n, cl = p->cl, q = n - 1;
  const cx *bs = inverse ? p->bI : p->bF;
  cx x0 = src[0];
  cx sum = mk(0, 0);
  for (int i = 0; i < n; i++) sum = cadd(sum, src[i]);
  cx *a = cxalloc(cl);
  for (int k = 0; k < q; k++) a[k] = src[p->perm[k]];
  or_plan *plan = cached_plan(cl);
  cx *A = cxalloc(cl);
  plan_fft(plan, A, a);
  for (int i = 0; i < cl; i++) A[i] = cmul(A[i], bs[i]);
  cx *conv = cxalloc(cl);
  plan_ifft(plan, conv, A);
  dst[0] = sum;
  int off = p->cyclic ? 0 : q;
  for (int qi = 0; qi < q; qi++) dst[p->iperm[qi]] = cadd(x0, conv[qi + off]);
  free(a);
  free(A);
  free(conv);
}

/* ---- Bluestein (bluestein.go, internal/kernels) -------------------------- */

/* internal/kernels/kernels.go:20-32 */
static void bit_reverse(cx *x, int n) {
  for (int i = 1, j = 0; i < n; i++) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) { cx t = x[i]; x[i] = x[j]; x[j] = t; }
  }
}

/* internal/kernels/kernels.go:38-59 (per-stage recurrence twiddles). */
static void radix2_recurrence(cx *x, int n, int inverse) {
  double sign = inverse ? 1.0 : -1.0;
  for (int len = 2; len <= n; len <<= 1) {
    double ang = sign * 2 * M_PI / (double)len;
    cx wlen = mk(cos(ang), sin(ang));
    int half = len >> 1;
    for (int start = 0; start < n; start += len) {
      cx w = mk(1, 0);
      for (int k = 0; k < half; k++) {
        cx u = x[start + k];
        cx v = cmul(x[start + k + half], w);
        x[start + k] = cadd(u, v);
        x[start + k + half] = csub(u, v);
        w = cmul(w, wlen);
      }
    }
  }
}

/* bluestein.go:52-63 */
static cx *bluestein_kernel(const cx *w, int n, int m) {
  cx *b = cxalloc(m);
  b[0] = cconj(w[0]);
  for (int j = 1; j < n; j++) {
    cx c = cconj(w[j]);
    b[j] = c;
    b[m - j] = c;
  }
  bit_reverse(b, m);
  radix2_recurrence(b, m, 0);
  return b;
}

int or_bluestein_m(int n) {
  int m = 1;
  while (m < 2 * n - 1) m <<= 1;
  return m;
}

void or_chirp_index(int n, int64_t *out) {
  for (int64_t j = 0; j < n; j++) out[j] = (j * j) % (2 * (int64_t)n);
}

/* bluestein.go:28-48 */
static blue_plan *new_blue_plan(int n) {
  blue_plan *p = (blue_plan *)calloc(1, sizeof(blue_plan));
  p->n = n;
  p->m = or_bluestein_m(n);
  p->wF = cxalloc(n);
  p->wI = cxalloc(n);
  for (int64_t j = 0; j < n; j++) {
    int64_t jj = (j * j) % (2 * (int64_t)n);
    double ang = M_PI * (double)jj / (double)n;
    p->wF[j] = mk(cos(-ang), sin(-ang));
    p->wI[j] = mk(cos(ang), sin(ang));
  }
  p->bF = bluestein_kernel(p->wF, n, p->m);
  p->bI = bluestein_kernel(p->wI, n, p->m);
  return p;
}

/* bluestein.go:67-95 */
static void blue_transform(blue_plan *p, cx *dst, const cx *src, int inverse) {
  int n = p->n, m = p->m;
  const cx *w = inverse ? p->wI : p->wF;
  const cx *bs = inverse ? p->bI : p->bF;
  cx *a = cxalloc(m);
  for (int j = 0; j < n; j++) a[j] = cmul(src[j], w[j]);
  bit_reverse(a, m);
  radix2_recurrence(a, m, 0);
  for (int i = 0; i < m; i++) a[i] = cmul(a[i], bs[i]);
  bit_reverse(a, m);
  radix2_recurrence(a, m, 1);
  cx inv = mk(1 / (double)m, 0);
  for (int i = 0; i < m; i++) a[i] = cmul(a[i], inv);
  for (int k = 0; k < n; k++) dst[k] = cmul(a[k], w[k]);
  free(a);
}

/* ---- Plan, router, cache (plan.go) -------------------------------------- */

/* plan.go:42-73 */
static or_plan *new_plan(int n) {
  or_plan *p = (or_plan *)calloc(1, sizeof(or_plan));
  p->n = n;
  switch (or_engine(n)) {
    case OR_IT: p->it = new_it_plan(n); break;
    case OR_CT: p->ct = new_ct_plan(n); break;
    case OR_RADER: p->rader = new_rader_plan(n); break;
    case OR_BLUESTEIN: p->blue = new_blue_plan(n); break;
    default: break;
  }
  return p;
}

/* plan.go:287-317: memo keyed by n, built outside the lock. */
#define CACHE_SLOTS 8192
static pthread_mutex_t plan_mu = PTHREAD_MUTEX_INITIALIZER;
static int cache_key[CACHE_SLOTS];
static or_plan *cache_val[CACHE_SLOTS];

static or_plan *cache_lookup(int n) {
  unsigned h = ((unsigned)n * 2654435761u) % CACHE_SLOTS;
  for (unsigned i = 0; i < CACHE_SLOTS; i++) {
    unsigned s = (h + i) % CACHE_SLOTS;
    if (!cache_val[s]) return NULL;
    if (cache_key[s] == n) return cache_val[s];
  }
  return NULL;
}

static or_plan *cache_store(int n, or_plan *p) {
  unsigned h = ((unsigned)n * 2654435761u) % CACHE_SLOTS;
  for (unsigned i = 0; i < CACHE_SLOTS; i++) {
    unsigned s = (h + i) % CACHE_SLOTS;
    if (!cache_val[s]) { cache_key[s] = n; cache_val[s] = p; return p; }
    if (cache_key[s] == n) return cache_val[s];
  }
  abort();
}

static or_plan *cached_plan(int n) {
  pthread_mutex_lock(&plan_mu);
  or_plan *p = cache_lookup(n);
  pthread_mutex_unlock(&plan_mu);
  if (p) return p;
  p = new_plan(n);
  pthread_mutex_lock(&plan_mu);
  or_plan *won = cache_store(n, p);
  pthread_mutex_unlock(&plan_mu);
  return won; /* the loser's plan is simply leaked, as the reference drops it */
}

/* plan.go:113-129 */
static void plan_execute(or_plan *p, cx *dst, const cx *src, int inverse) {
  int n = p->n;
  if (n <= 1) {
    if (n == 1 && dst != src) dst[0] = src[0];
    return;
  }
  if (p->it) it_transform(p->it, dst, src, inverse);
  else if (p->ct) ct_transform(p->ct, dst, src, inverse);
  else if (p->rader) rader_transform(p->rader, dst, src, inverse);
  else blue_transform(p->blue, dst, src, inverse);
}

/* plan.go:91-94 */
static void plan_fft(or_plan *p, cx *dst, const cx *src) { plan_execute(p, dst, src, 0); }

/* plan.go:98-109 */
static void plan_ifft(or_plan *p, cx *dst, const cx *src) {
  plan_execute(p, dst, src, 1);
  int n = p->n;
  if (n == 0) return;
  cx inv = mk(1 / (double)n, 0);
  for (int i = 0; i < n; i++) dst[i] = cmul(dst[i], inv);
}

void or_execute(int n, double *dst, const double *src, int inverse) {
  plan_execute(cached_plan(n), (cx *)dst, (const cx *)src, inverse);
}
void or_fft(int n, double *dst, const double *src) {
  plan_fft(cached_plan(n), (cx *)dst, (const cx *)src);
}
void or_ifft(int n, double *dst, const double *src) {
  plan_ifft(cached_plan(n), (cx *)dst, (const cx *)src);
}

void or_bluestein_transform(int n, double *dst, const double *src, int inverse) {
  blue_plan *p = new_blue_plan(n);
  blue_transform(p, (cx *)dst, (const cx *)src, inverse);
  free(p->wF); free(p->wI); free(p->bF); free(p->bI); free(p);
}

void or_rader_transform(int n, double *dst, const double *src, int inverse) {
  rader_plan *p = new_rader_plan(n);
  cx *tmp = NULL;
  if (dst == src) {
    tmp = cxalloc(n);
    memcpy(tmp, src, sizeof(cx) * n);
    src = (const double *)tmp;
  }
  rader_transform(p, (cx *)dst, (const cx *)src, inverse);
  free(tmp);
  free(p->perm); free(p->iperm); free(p->bF); free(p->bI); free(p);
}

int or_rader_info(int n, int *cyclic, int *g, int *perm, int *iperm) {
  int q = n - 1;
  int gg = or_primitive_root(n);
  int cyc = or_factors_small(q);
  int cl = cyc ? q : or_best_conv_len(2 * q);
  if (cyclic) *cyclic = cyc;
  if (g) *g = gg;
  if (perm && iperm) {
    int64_t x = 1;
    for (int k = 0; k < q; k++) { perm[k] = (int)x; x = x * gg % n; }
    for (int qi = 0; qi < q; qi++) iperm[qi] = perm[(q - qi) % q];
  }
  return cl;
}

/* ======================================================================== */
/* Real transforms (realplan.go, rfft.go)                                    */
/* ======================================================================== */

typedef struct {
  int n;
  or_plan *half; /* even path */
  cx *tw;        /* W_n^k, k = 0..n/2 */
  or_plan *full; /* odd / trivial path */
} real_plan;

/* realplan.go:37-58 */
static real_plan *new_real_plan(int n) {
  real_plan *p = (real_plan *)calloc(1, sizeof(real_plan));
  p->n = n;
  if (n <= 1 || n % 2 != 0) {
    if (n >= 1) p->full = cached_plan(n);
    return p;
  }
  int m = n / 2;
  p->half = cached_plan(m);
  p->tw = cxalloc(m + 1);
  for (int k = 0; k <= m; k++) {
    double ang = -2 * M_PI * (double)k / (double)n;
    p->tw[k] = mk(cos(ang), sin(ang));
  }
  return p;
}

static pthread_mutex_t real_mu = PTHREAD_MUTEX_INITIALIZER;
static int rcache_key[CACHE_SLOTS];
static real_plan *rcache_val[CACHE_SLOTS];

/* rfft.go:55-64: this cache builds under the lock (the reference does). */
static real_plan *cached_real_plan(int n) {
  pthread_mutex_lock(&real_mu);
  unsigned h = ((unsigned)n * 2654435761u) % CACHE_SLOTS;
  real_plan *p = NULL;
  for (unsigned i = 0; i < CACHE_SLOTS; i++) {
    unsigned s = (h + i) % CACHE_SLOTS;
    if (!rcache_val[s]) {
      p = new_real_plan(n);
      rcache_key[s] = n;
      rcache_val[s] = p;
      break;
    }
    if (rcache_key[s] == n) { p = rcache_val[s]; break; }
  }
  pthread_mutex_unlock(&real_mu);
  return p;
}

/* realplan.go:138-169 */
static void rfft_untangle(cx *dst, const cx *Z, const cx *tw, int m) {
  double z0r = Z[0].re, z0i = Z[0].im;
  dst[0] = mk(z0r + z0i, 0);
  dst[m] = mk(z0r - z0i, 0);
  int half = (m - 1) / 2;
  for (int k = 1; k <= half; k++) {
    cx zk = Z[k], zmk = Z[m - k];
    double xer = (zk.re + zmk.re) * 0.5;
    double xei = (zk.im - zmk.im) * 0.5;
    double xor_ = (zk.im + zmk.im) * 0.5;
    double xoi = -(zk.re - zmk.re) * 0.5;
    double wr = tw[k].re, wi = tw[k].im;
    double tr = wr * xor_ - wi * xoi;
    double ti = wr * xoi + wi * xor_;
    dst[k] = mk(xer + tr, xei + ti);
    dst[m - k] = mk(xer - tr, -(xei - ti));
  }
  if ((m & 1) == 0) {
    int k = m / 2;
    dst[k] = mk(Z[k].re, -Z[k].im);
  }
}

/* realplan.go:77-116 */
static void real_rfft(real_plan *p, cx *dst, const double *src) {
  int n = p->n;
  if (n == 0) return;
  if (n == 1) { dst[0] = mk(src[0], 0); return; }
  if (!p->half) {
    cx *c = cxalloc(n), *full = cxalloc(n);
    for (int i = 0; i < n; i++) c[i] = mk(src[i], 0);
    plan_fft(p->full, full, c);
    memcpy(dst, full, sizeof(cx) * (n / 2 + 1));
    free(c);
    free(full);
    return;
  }
  int m = n / 2;
  cx *z = cxalloc(m), *Z = cxalloc(m);
  if (p->half->it) {
    it_transform_real_packed(p->half->it, Z, src);
  } else {
    for (int j = 0; j < m; j++) z[j] = mk(src[2 * j], src[2 * j + 1]);
    plan_fft(p->half, Z, z);
  }
  rfft_untangle(dst, Z, p->tw, m);
  free(z);
  free(Z);
}

/* realplan.go:197-213 */
static void irfft_full(real_plan *p, double *dst, const cx *src, int nsrc) {
  int n = p->n;
  cx *full = cxalloc(n);
  int half = n / 2 + 1;
  for (int k = 0; k < half && k < nsrc; k++) {
    full[k] = src[k];
    if (k > 0 && k < n - k) full[n - k] = cconj(src[k]);
  }
  cx *inv = cxalloc(n);
  plan_ifft(cached_plan(n), inv, full);
  for (int i = 0; i < n; i++) dst[i] = inv[i].re;
  free(full);
  free(inv);
}

/* realplan.go:221-296 */
static void irfft_packed(real_plan *p, double *dst, const cx *src, int nsrc) {
  int n = p->n, m = n / 2;
#define BIN(k) ((k) < nsrc ? src[(k)] : mk(0, 0))
  cx *z = cxalloc(m), *Z = cxalloc(m);
  double x0 = BIN(0).re, xm = BIN(m).re;
  Z[0] = mk((x0 + xm) * 0.5, (x0 - xm) * 0.5);
  for (int k = 1; k <= m - k; k++) {
    cx xk = BIN(k), xmk = BIN(m - k);
    cx cmk = cconj(xmk);
    double xer = (xk.re + cmk.re) * 0.5;
    double xei = (xk.im + cmk.im) * 0.5;
    double dr = (xk.re - cmk.re) * 0.5;
    double di = (xk.im - cmk.im) * 0.5;
    double wr = p->tw[k].re, wi = p->tw[k].im;
    double xor_ = wr * dr + wi * di;
    double xoi = wr * di - wi * dr;
    Z[k] = mk(xer - xoi, xei + xor_);
    if (k != m - k) Z[m - k] = mk(xer + xoi, -(xei - xor_));
  }
#undef BIN
  if (p->half->it) {
    it_transform_scratch(p->half->it, z, Z, 1);
    double inv = 1 / (double)m;
    for (int j = 0; j < m; j++) {
      dst[2 * j] = z[j].re * inv;
      dst[2 * j + 1] = z[j].im * inv;
    }
  } else {
    plan_ifft(p->half, z, Z);
    for (int j = 0; j < m; j++) {
      dst[2 * j] = z[j].re;
      dst[2 * j + 1] = z[j].im;
    }
  }
  free(z);
  free(Z);
}

/* realplan.go:181-192 */
static void real_irfft(real_plan *p, double *dst, const cx *src, int nsrc) {
  if (p->n <= 0) return;
  if (!p->half) irfft_full(p, dst, src, nsrc);
  else irfft_packed(p, dst, src, nsrc);
}

void or_rfft(int n, double *dst, const double *src) {
  if (n == 0) return;
  real_rfft(cached_real_plan(n), (cx *)dst, src);
}

void or_irfft(int n, double *dst, const double *src, int nsrc) {
  if (n <= 0) return;
  real_irfft(cached_real_plan(n), dst, (const cx *)src, nsrc);
}

/* ======================================================================== */
/* Goroutine fan-out (parallel.go) as a pthread pool                          */
/* ======================================================================== */

static int par_workers = 0;
#define PAR_THRESHOLD (1 << 14)

void or_set_workers(int w) { par_workers = w; }
int or_get_workers(void) {
  if (par_workers <= 0) {
    long c = sysconf(_SC_NPROCESSORS_ONLN);
    par_workers = c > 0 ? (int)c : 1;
  }
  return par_workers;
}

typedef void (*chunk_fn)(void *ctx, int64_t lo, int64_t hi);
typedef struct { chunk_fn fn; void *ctx; int64_t lo, hi; } chunk_job;

static void *chunk_thread(void *arg) {
  chunk_job *j = (chunk_job *)arg;
  j->fn(j->ctx, j->lo, j->hi);
  return NULL;
}

/* parallel.go:32-55 */
static void par_chunks(int64_t n, chunk_fn fn, void *ctx) {
  int64_t w = or_get_workers();
  if (w > n) w = n;
  if (w <= 1) { fn(ctx, 0, n); return; }
  int64_t chunk = (n + w - 1) / w;
  int64_t cnt = (n + chunk - 1) / chunk;
  pthread_t *th = (pthread_t *)xmalloc(sizeof(pthread_t) * cnt);
  chunk_job *jobs = (chunk_job *)xmalloc(sizeof(chunk_job) * cnt);
  int64_t c = 0;
  for (int64_t lo = 0; lo < n; lo += chunk, c++) {
    int64_t hi = lo + chunk < n ? lo + chunk : n;
    jobs[c].fn = fn; jobs[c].ctx = ctx; jobs[c].lo = lo; jobs[c].hi = hi;
    pthread_create(&th[c], NULL, chunk_thread, &jobs[c]);
  }
  for (int64_t i = 0; i < cnt; i++) pthread_join(th[i], NULL);
  free(th);
  free(jobs);
}

/* parallel.go:59-61 */
static int parallelize_lines(int64_t count, int64_t len) {
  return or_get_workers() > 1 && count > 1 && count * len >= PAR_THRESHOLD;
}

static void run_lines(int64_t count, int64_t len, chunk_fn fn, void *ctx) {
  if (parallelize_lines(count, len)) par_chunks(count, fn, ctx);
  else fn(ctx, 0, count);
}

/* ======================================================================== */
/* N-D (ndfft.go)                                                             */
/* ======================================================================== */

/* ndfft.go:144-155 */
static int64_t line_base(int64_t c, const int *shape, const int64_t *stride, int rank, int ax) {
  int64_t base = 0;
  for (int a = rank - 1; a >= 0; a--) {
    if (a == ax) continue;
    int64_t s = shape[a];
    base += (c % s) * stride[a];
    c /= s;
  }
  return base;
}

typedef struct {
  cx *out;
  const int *shape;
  const int64_t *stride;
  int rank, ax, inverse;
  or_plan *plan;
} axis_ctx;

static void axis_work(void *vctx, int64_t lo, int64_t hi) {
  axis_ctx *c = (axis_ctx *)vctx;
  int n = c->shape[c->ax];
  int64_t st = c->stride[c->ax];
  cx *buf = cxalloc(n), *res = cxalloc(n);
  for (int64_t l = lo; l < hi; l++) {
    int64_t base = line_base(l, c->shape, c->stride, c->rank, c->ax);
    for (int i = 0; i < n; i++) buf[i] = c->out[base + i * st];
    if (c->inverse) plan_ifft(c->plan, res, buf);
    else plan_fft(c->plan, res, buf);
    for (int i = 0; i < n; i++) c->out[base + i * st] = res[i];
  }
  free(buf);
  free(res);
}

/* ndfft.go:102-136 */
static void transform_axis(cx *out, int64_t total, const int *shape, const int64_t *stride, int rank,
                           int ax, int inverse) {
  int n = shape[ax];
  if (n == 1) return;
  axis_ctx c = {out, shape, stride, rank, ax, inverse, cached_plan(n)};
  run_lines(total / n, n, axis_work, &c);
}

/* ndfft.go:66-90 (shape validated by the caller). */
void or_fftn(double *outd, const double *data, const int *shape, int rank, int inverse) {
  int64_t total = 1;
  for (int a = 0; a < rank; a++) total *= shape[a];
  cx *out = (cx *)outd;
  if ((const double *)out != data) memcpy(out, data, sizeof(cx) * total);
  if (total <= 1) return;
  int64_t stride[32];
  int64_t acc = 1;
  for (int a = rank - 1; a >= 0; a--) { stride[a] = acc; acc *= shape[a]; }
  for (int a = 0; a < rank; a++) transform_axis(out, total, shape, stride, rank, a, inverse);
}

/* ======================================================================== */
/* Real 2-D (rfft2.go)                                                        */
/* ======================================================================== */

typedef struct {
  const double *data;
  cx *half;
  double *out;
  int rows, cols, rcols, inverse;
  real_plan *rp;
  or_plan *cp;
} r2_ctx;

static void r2_row_fwd(void *v, int64_t lo, int64_t hi) {
  r2_ctx *c = (r2_ctx *)v;
  double *row = (double *)xmalloc(sizeof(double) * c->cols);
  cx *dst = cxalloc(c->rcols);
  for (int64_t r = lo; r < hi; r++) {
    memcpy(row, c->data + r * c->cols, sizeof(double) * c->cols);
    real_rfft(c->rp, dst, row);
    memcpy(c->half + r * c->rcols, dst, sizeof(cx) * c->rcols);
  }
  free(row);
  free(dst);
}

static void r2_col(void *v, int64_t lo, int64_t hi) {
  r2_ctx *c = (r2_ctx *)v;
  cx *col = cxalloc(c->rows), *dst = cxalloc(c->rows);
  for (int64_t k = lo; k < hi; k++) {
    for (int r = 0; r < c->rows; r++) col[r] = c->half[(int64_t)r * c->rcols + k];
    if (c->inverse) plan_ifft(c->cp, dst, col);
    else plan_fft(c->cp, dst, col);
    for (int r = 0; r < c->rows; r++) c->half[(int64_t)r * c->rcols + k] = dst[r];
  }
  free(col);
  free(dst);
}

static void r2_row_inv(void *v, int64_t lo, int64_t hi) {
  r2_ctx *c = (r2_ctx *)v;
  double *dst = (double *)xmalloc(sizeof(double) * c->cols);
  for (int64_t r = lo; r < hi; r++) {
    real_irfft(c->rp, dst, c->half + r * c->rcols, c->rcols);
    memcpy(c->out + r * c->cols, dst, sizeof(double) * c->cols);
  }
  free(dst);
}

/* rfft2.go:22-74 */
void or_rfft2(double *out, const double *data, int rows, int cols) {
  int rcols = cols / 2 + 1;
  r2_ctx c = {data, (cx *)out, NULL, rows, cols, rcols, 0, cached_real_plan(cols), NULL};
  run_lines(rows, cols, r2_row_fwd, &c);
  c.cp = cached_plan(rows);
  run_lines(rcols, rows, r2_col, &c);
}

/* rfft2.go:87-138 */
void or_irfft2(double *out, const double *data, int64_t ndata, int rows, int cols) {
  int rcols = cols / 2 + 1;
  int64_t tot = (int64_t)rows * rcols;
  cx *half = cxalloc(tot);
  for (int64_t i = 0; i < tot && i < ndata; i++) half[i] = ((const cx *)data)[i];
  r2_ctx c = {NULL, half, out, rows, cols, rcols, 1, NULL, cached_plan(rows)};
  run_lines(rcols, rows, r2_col, &c);
  c.rp = cached_real_plan(cols);
  run_lines(rows, cols, r2_row_inv, &c);
  free(half);
}

/* ======================================================================== */
/* Spectral helpers (freq.go, window.go)                                      */
/* ======================================================================== */

/* window.go:59-78 */
void or_cosine_window(int n, const double *a, int na, double *w) {
  if (n <= 0) return;
  if (n == 1) { w[0] = 1; return; }
  double denom = (double)(n - 1);
  for (int k = 0; k < n; k++) {
    double s = a[0], sign = -1.0;
    for (int j = 1; j < na; j++) {
      s += sign * a[j] * cos(2 * M_PI * (double)j * (double)k / denom);
      sign = -sign;
    }
    w[k] = s;
  }
}

/* window.go:20-22 */
void or_hann(int n, double *out) {
  static const double a[2] = {0.5, 0.5};
  or_cosine_window(n, a, 2, out);
}

/* freq.go:69-90 */
void or_psd(int n, const double *x, double d, double *out) {
  if (n == 0) return;
  int m = n / 2 + 1;
  cx *spec = cxalloc(m);
  real_rfft(cached_real_plan(n), spec, x);
  double scale = d / (double)n;
  for (int k = 0; k < m; k++) {
    double re = spec[k].re, im = spec[k].im;
    double p = (re * re + im * im) * scale;
    if (k != 0 && !(n % 2 == 0 && k == m - 1)) p *= 2;
    out[k] = p;
  }
  free(spec);
}

/* freq.go:107-127 (argument checks are the caller's). */
int or_spectrogram(const double *x, int64_t nx, int segment, int overlap, const double *window,
                   double d, double *out) {
  int step = segment - overlap;
  int bins = segment / 2 + 1;
  double *seg = (double *)xmalloc(sizeof(double) * segment);
  int frames = 0;
  for (int64_t start = 0; start + segment <= nx; start += step) {
    if (out) {
      for (int i = 0; i < segment; i++) seg[i] = x[start + i] * window[i];
      or_psd(segment, seg, d, out + (int64_t)frames * bins);
    }
    frames++;
  }
  free(seg);
  return frames;
}

/* ======================================================================== */
/* Batch helpers for the CPU baseline                                         */
/* ======================================================================== */

typedef struct { int n, inverse; cx *dst; const cx *src; or_plan *p; } batch_ctx;

static void batch_work(void *v, int64_t lo, int64_t hi) {
  batch_ctx *c = (batch_ctx *)v;
  for (int64_t b = lo; b < hi; b++) {
    if (c->inverse) plan_ifft(c->p, c->dst + b * c->n, c->src + b * c->n);
    else plan_fft(c->p, c->dst + b * c->n, c->src + b * c->n);
  }
}

void or_batch_fft(int n, int64_t batch, double *dst, const double *src, int inverse) {
  batch_ctx c = {n, inverse, (cx *)dst, (const cx *)src, cached_plan(n)};
  if (or_get_workers() > 1 && batch > 1) par_chunks(batch, batch_work, &c);
  else batch_work(&c, 0, batch);
}

void or_batch_rfft2_roundtrip(int64_t batch, int rows, int cols, const double *x, double *spec,
                              double *back) {
  int64_t in_sz = (int64_t)rows * cols, sp_sz = (int64_t)rows * (cols / 2 + 1);
  for (int64_t b = 0; b < batch; b++) {
    or_rfft2(spec + b * sp_sz * 2, x + b * in_sz, rows, cols);
    or_irfft2(back + b * in_sz, spec + b * sp_sz * 2, sp_sz, rows, cols);
  }
}
