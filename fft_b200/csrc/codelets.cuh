// codelets.cuh -- straight-line forward DFT-R kernels on registers.
//
// All codelets compute X[k] = sum_n v[n] exp(-2 pi i n k / R) in place on an
// array of R complex values.  The inverse transform is never coded separately:
// the engine conjugates on load and on store (IDFT(x) = conj(DFT(conj(x)))).
//
// Radix 2/4/8/16/32 are the power-of-two building blocks (16 = 4 x 4 and
// 32 = 4 x 8 with their twiddles as constants); odd primes R in {3,5,7,11,13} share one
// conjugate-pair template: with s_q = v_q + v_{R-q}, d_q = v_q - v_{R-q},
//   X[k]   = v0 + sum_q cos(2 pi q k / R) s_q - i sum_q sin(2 pi q k / R) d_q
//   X[R-k] = v0 + sum_q cos(2 pi q k / R) s_q + i sum_q sin(2 pi q k / R) d_q
// for k = 1..(R-1)/2.  The trigonometric constants are values of cos/sin at
// rational multiples of 2 pi, written to 25 significant digits.
#pragma once
#include "common.cuh"

namespace gf {

// cos(2 pi m / R) and sin(2 pi m / R) for m = 1..(R-1)/2 and the odd primes.
GF_HD constexpr double ctab(int R, int m) {
  return R == 3 ? -0.5
       : R == 5 ? (m == 1 ? 0.3090169943749474241022934 : -0.8090169943749474241022934)
       : R == 7 ? (m == 1 ? 0.6234898018587335305250049
                 : m == 2 ? -0.2225209339563144042889026 : -0.9009688679024191262361023)
       : R == 11 ? (m == 1 ? 0.8412535328311811688618116
                  : m == 2 ? 0.4154150130018864255292741
                  : m == 3 ? -0.1423148382732851404437927
                  : m == 4 ? -0.6548607339452850640569251 : -0.9594929736144973898903681)
       : /* 13 */ (m == 1 ? 0.8854560256532098959003755
                  : m == 2 ? 0.5680647467311558025118076
                  : m == 3 ? 0.1205366802553230533490677
                  : m == 4 ? -0.3546048870425356259696379
                  : m == 5 ? -0.7485107481711010986346306 : -0.9709418174260520271569823);
}
GF_HD constexpr double stab(int R, int m) {
  return R == 3 ? 0.8660254037844386467637232
       : R == 5 ? (m == 1 ? 0.9510565162951535721164393 : 0.5877852522924731291687060)
       : R == 7 ? (m == 1 ? 0.7818314824680298087084445
                 : m == 2 ? 0.9749279121818236070181317 : 0.4338837391175581204757683)
       : R == 11 ? (m == 1 ? 0.5406408174555975821076360
                  : m == 2 ? 0.9096319953545183714117154
                  : m == 3 ? 0.9898214418809327323760920
                  : m == 4 ? 0.7557495743542582837740358 : 0.2817325568414296977114179)
       : /* 13 */ (m == 1 ? 0.4647231720437685456560153
                  : m == 2 ? 0.8229838658936563945796174
                  : m == 3 ? 0.9927088740980539928007516
                  : m == 4 ? 0.9350162426854148234397846
                  : m == 5 ? 0.6631226582407952023767855 : 0.2393156642875577671487537);
}
// cos/sin(2 pi e / R) for any integer e, folded into the first half-period.
GF_HD constexpr double cosr(int R, int e) {
  return (e % R) == 0 ? 1.0 : ((e % R) <= R / 2 ? ctab(R, e % R) : ctab(R, R - e % R));
}
GF_HD constexpr double sinr(int R, int e) {
  return (e % R) == 0 ? 0.0 : ((e % R) <= R / 2 ? stab(R, e % R) : -stab(R, R - e % R));
}

constexpr double kSqrtHalf = 0.7071067811865475244008444;
constexpr double kCos8 = 0.9238795325112867561281832;  // cos(pi/8)
constexpr double kSin8 = 0.3826834323650897717284600;  // sin(pi/8)

template <class C> GF_DEV void dft2(C &a, C &b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

// In-place DFT-4 on (a,b,c,d) = v[0..3] (forward).
template <class C> GF_DEV void dft4(C &a, C &b, C &c, C &d) {
  C t0 = cadd(a, c), t1 = csub(a, c);
  C t2 = cadd(b, d), t3 = cmul_mi(csub(b, d));
  a = cadd(t0, t2);
  c = csub(t0, t2);
  b = cadd(t1, t3);
  d = csub(t1, t3);
}

template <class C> GF_DEV C mul_w8_1(C z) {  // z * exp(-i pi/4)
  using R = decltype(z.x);
  const R h = (R)kSqrtHalf;
  return mkc((z.x + z.y) * h, (z.y - z.x) * h);
}
template <class C> GF_DEV C mul_w8_3(C z) {  // z * exp(-3 i pi/4)
  using R = decltype(z.x);
  const R h = (R)kSqrtHalf;
  return mkc((z.y - z.x) * h, -(z.x + z.y) * h);
}

template <int R, class C> struct Dft;

template <class C> struct Dft<2, C> {
  static GF_DEV void run(C *v) { dft2(v[0], v[1]); }
};
template <class C> struct Dft<4, C> {
  static GF_DEV void run(C *v) { dft4(v[0], v[1], v[2], v[3]); }
};

// DFT-8 as 2 x 4: butterflies n, n+4 with twiddles W8^n, then two DFT-4.
template <class C> struct Dft<8, C> {
  static GF_DEV void run(C *v) {
    C a0 = cadd(v[0], v[4]), b0 = csub(v[0], v[4]);
    C a1 = cadd(v[1], v[5]), b1 = mul_w8_1(csub(v[1], v[5]));
    C a2 = cadd(v[2], v[6]), b2 = cmul_mi(csub(v[2], v[6]));
    C a3 = cadd(v[3], v[7]), b3 = mul_w8_3(csub(v[3], v[7]));
    dft4(a0, a1, a2, a3);
    dft4(b0, b1, b2, b3);
    v[0] = a0; v[2] = a1; v[4] = a2; v[6] = a3;
    v[1] = b0; v[3] = b1; v[5] = b2; v[7] = b3;
  }
};

// DFT-16 as 4 x 4: n = n1 + 4 n2, k = k2 + 4 k1.
template <class C> struct Dft<16, C> {
  static GF_DEV void run(C *v) {
    using Rl = decltype(v[0].x);
    const Rl c8 = (Rl)kCos8, s8 = (Rl)kSin8, h = (Rl)kSqrtHalf;
    C y[16];
#pragma unroll
    for (int n1 = 0; n1 < 4; n1++) {
      C a = v[n1], b = v[n1 + 4], c = v[n1 + 8], d = v[n1 + 12];
      dft4(a, b, c, d);
      y[n1 * 4 + 0] = a; y[n1 * 4 + 1] = b; y[n1 * 4 + 2] = c; y[n1 * 4 + 3] = d;
    }
    // twiddles W16^(n1*k2)
    // n1=1: W^1, W^2, W^3 ; n1=2: W^2, W^4, W^6 ; n1=3: W^3, W^6, W^9
    // W16^1 = (c8, -s8), W16^2 = (h, -h), W16^3 = (s8, -c8), W16^4 = -i,
    // W16^6 = (-h, -h), W16^9 = (-c8, s8)
    y[5] = cmul(y[5], mkc(c8, -s8));
    y[6] = mul_w8_1(y[6]);
    y[7] = cmul(y[7], mkc(s8, -c8));
    y[9] = mul_w8_1(y[9]);
    y[10] = cmul_mi(y[10]);
    y[11] = mul_w8_3(y[11]);
    y[13] = cmul(y[13], mkc(s8, -c8));
    y[14] = mul_w8_3(y[14]);
    y[15] = cmul(y[15], mkc(-c8, s8));
    (void)h;
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) {
      C a = y[k2], b = y[4 + k2], c = y[8 + k2], d = y[12 + k2];
      dft4(a, b, c, d);
      v[k2] = a; v[k2 + 4] = b; v[k2 + 8] = c; v[k2 + 12] = d;
    }
  }
};

// cos(pi e / 16) and sin(pi e / 16) for any integer e (the W32 constants).
GF_HD constexpr double cos16(int e) {
  constexpr double t[9] = {1.0,
                           0.9807852804032304491261822,
                           0.9238795325112867561281832,
                           0.8314696123025452370787884,
                           0.7071067811865475244008444,
                           0.5555702330196022247428308,
                           0.3826834323650897717284600,
                           0.1950903220161282678482849,
                           0.0};
  return ((e % 32) + 32) % 32 <= 8    ? t[((e % 32) + 32) % 32]
         : ((e % 32) + 32) % 32 <= 16 ? -t[16 - ((e % 32) + 32) % 32]
         : ((e % 32) + 32) % 32 <= 24 ? -t[((e % 32) + 32) % 32 - 16]
                                      : t[32 - ((e % 32) + 32) % 32];
}
GF_HD constexpr double sin16(int e) { return cos16(8 - e); }

// z * W32^e = z * exp(-2 pi i e / 32), with the trivial angles folded.
template <int E, class C> GF_DEV C tw32(C z) {
  using Rl = decltype(z.x);
  constexpr int e = ((E % 32) + 32) % 32;
  if constexpr (e == 0) return z;
  else if constexpr (e == 8) return cmul_mi(z);
  else if constexpr (e == 16) return mkc(-z.x, -z.y);
  else if constexpr (e == 24) return cmul_pi(z);
  else if constexpr (e == 4) return mul_w8_1(z);
  else if constexpr (e == 12) return mul_w8_3(z);
  else return cmul(z, mkc((Rl)cos16(e), (Rl)-sin16(e)));
}

// DFT-32 as 4 x 8: n = n1 + 4 n2, k = k2 + 8 k1; DFT-8 over n2 for each n1,
// twiddles W32^(n1 k2), DFT-4 over n1 for each k2.
template <int N1, class C> GF_DEV void dft32_col(C *v, C (&y)[32]) {
  C t[8];
#pragma unroll
  for (int n2 = 0; n2 < 8; n2++) t[n2] = v[N1 + 4 * n2];
  Dft<8, C>::run(t);
  y[N1 * 8 + 0] = t[0];
  y[N1 * 8 + 1] = tw32<N1 * 1>(t[1]);
  y[N1 * 8 + 2] = tw32<N1 * 2>(t[2]);
  y[N1 * 8 + 3] = tw32<N1 * 3>(t[3]);
  y[N1 * 8 + 4] = tw32<N1 * 4>(t[4]);
  y[N1 * 8 + 5] = tw32<N1 * 5>(t[5]);
  y[N1 * 8 + 6] = tw32<N1 * 6>(t[6]);
  y[N1 * 8 + 7] = tw32<N1 * 7>(t[7]);
}
template <class C> struct Dft<32, C> {
  static GF_DEV void run(C *v) {
    C y[32];
    dft32_col<0>(v, y);
    dft32_col<1>(v, y);
    dft32_col<2>(v, y);
    dft32_col<3>(v, y);
#pragma unroll
    for (int k2 = 0; k2 < 8; k2++) {
      C a = y[k2], b = y[8 + k2], c = y[16 + k2], d = y[24 + k2];
      dft4(a, b, c, d);
      v[k2] = a; v[k2 + 8] = b; v[k2 + 16] = c; v[k2 + 24] = d;
    }
  }
};

// Odd prime radix via conjugate pairs.
template <int R, class C> struct DftOdd {
  static GF_DEV void run(C *v) {
    using Rl = decltype(v[0].x);
    constexpr int H = (R - 1) / 2;
    C s[H], d[H];
    C x0 = v[0];
    C dc = x0;
#pragma unroll
    for (int q = 1; q <= H; q++) {
      s[q - 1] = cadd(v[q], v[R - q]);
      d[q - 1] = csub(v[q], v[R - q]);
      dc = cadd(dc, s[q - 1]);
    }
    v[0] = dc;
#pragma unroll
    for (int k = 1; k <= H; k++) {
      Rl ar = x0.x, ai = x0.y, br = 0, bi = 0;
#pragma unroll
      for (int q = 1; q <= H; q++) {
        const Rl cq = (Rl)cosr(R, q * k);
        const Rl sq = (Rl)sinr(R, q * k);
        ar += cq * s[q - 1].x;
        ai += cq * s[q - 1].y;
        br += sq * d[q - 1].x;
        bi += sq * d[q - 1].y;
      }
      // X[k] = A - i B, X[R-k] = A + i B
      v[k] = mkc(ar + bi, ai - br);
      v[R - k] = mkc(ar - bi, ai + br);
    }
  }
};
template <class C> struct Dft<3, C> : DftOdd<3, C> {};
template <class C> struct Dft<5, C> : DftOdd<5, C> {};
template <class C> struct Dft<7, C> : DftOdd<7, C> {};
template <class C> struct Dft<11, C> : DftOdd<11, C> {};
template <class C> struct Dft<13, C> : DftOdd<13, C> {};

}  // namespace gf
