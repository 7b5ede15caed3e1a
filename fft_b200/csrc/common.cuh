// common.cuh -- precision traits, complex helpers and fast integer division
// for the B200 line-FFT engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define GF_DEV __device__ __forceinline__
#define GF_HD __host__ __device__ __forceinline__

// ---------------------------------------------------------------------------
// Precision traits.  Every kernel is instantiated for three arithmetic forms:
//   PrecF64  -- complex128 data, FP64 twiddles (the parity form),
//   PrecF32  -- complex64 data, twiddles rounded once from FP64 to FP32,
//   PrecF32C -- complex64 data, FP64 twiddles kept as an FP32 hi+lo pair and
//               applied with a compensated product a*hi + a*lo.
// ---------------------------------------------------------------------------
struct PrecF64 {
  using real = double;
  using cpx = double2;
  using tw_t = double2;  // twiddle table entry
  using sp_t = double2;  // FP64 spectrum entry (Rader/Bluestein kernels)
  static constexpr int id = 0;
};
struct PrecF32 {
  using real = float;
  using cpx = float2;
  using tw_t = float2;
  using sp_t = float4;  // spectra always kept as hi+lo pairs
  static constexpr int id = 1;
};
struct PrecF32C {
  using real = float;
  using cpx = float2;
  using tw_t = float4;  // (hi.re, hi.im, lo.re, lo.im)
  using sp_t = float4;
  static constexpr int id = 2;
};

GF_DEV double2 mkc(double re, double im) { return make_double2(re, im); }
GF_DEV float2 mkc(float re, float im) { return make_float2(re, im); }

template <class C> GF_DEV C cadd(C a, C b) { return mkc(a.x + b.x, a.y + b.y); }
template <class C> GF_DEV C csub(C a, C b) { return mkc(a.x - b.x, a.y - b.y); }
template <class C> GF_DEV C cconj(C a) { return mkc(a.x, -a.y); }
// a * (-i)
template <class C> GF_DEV C cmul_mi(C a) { return mkc(a.y, -a.x); }
// a * (+i)
template <class C> GF_DEV C cmul_pi(C a) { return mkc(-a.y, a.x); }

GF_DEV double2 cmul(double2 a, double2 b) {
  return mkc(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
GF_DEV float2 cmul(float2 a, float2 b) {
  return mkc(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
template <class C, class R> GF_DEV C cscale(C a, R s) { return mkc(a.x * s, a.y * s); }

// Twiddle application in each precision form.
GF_DEV double2 twmul(double2 a, double2 w) { return cmul(a, w); }
GF_DEV float2 twmul(float2 a, float2 w) { return cmul(a, w); }
// Compensated: a*(hi+lo) = a*hi + a*lo, with the small a*lo term folded into
// the fused multiply-adds of the large one.
GF_DEV float2 twmul(float2 a, float4 w) {
  float re = fmaf(a.x, w.z, -a.y * w.w);
  float im = fmaf(a.x, w.w, a.y * w.z);
  re = fmaf(a.x, w.x, fmaf(-a.y, w.y, re));
  im = fmaf(a.x, w.y, fmaf(a.y, w.x, im));
  return mkc(re, im);
}
// Cache-hinted global loads.  Line data is read once per pass: it is not
// allocated in L1 (ld_stream), so the small tables every line rereads
// (stage twiddles, untangle roots) keep their L1 lines; those tables are
// read-only for the kernel's lifetime and loaded with L1 priority (ld_keep).
GF_DEV double2 ld_stream(const double2 *p) {
  double2 v;
  asm("ld.global.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
GF_DEV float2 ld_stream(const float2 *p) {
  float2 v;
  asm("ld.global.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
GF_DEV double ld_stream(const double *p) {
  double v;
  asm("ld.global.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
GF_DEV float ld_stream(const float *p) {
  float v;
  asm("ld.global.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
GF_DEV double ld_keep(const double *p) {
  double v;
  asm("ld.global.nc.L1::evict_last.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
GF_DEV float ld_keep(const float *p) {
  float v;
  asm("ld.global.nc.L1::evict_last.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
GF_DEV double2 ld_keep(const double2 *p) {
  double2 v;
  asm("ld.global.nc.L1::evict_last.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
GF_DEV float2 ld_keep(const float2 *p) {
  float2 v;
  asm("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}
GF_DEV float4 ld_keep(const float4 *p) {
  float4 v;
  asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p));
  return v;
}

// Spectrum multiply (Rader / Bluestein convolution): always FP64-derived.
GF_DEV double2 spmul(double2 a, double2 w) { return cmul(a, w); }
GF_DEV float2 spmul(float2 a, float4 w) { return twmul(a, w); }

// ---------------------------------------------------------------------------
// Unsigned division by a runtime-invariant divisor d (Granlund-Montgomery
// round-up method): with p = 31 + ceil(log2 d) and m = ceil(2^p / d) (which
// fits in 32 bits), q = (n * m) >> p is exact for every n < 2^31.
// ---------------------------------------------------------------------------
struct FastDiv {
  uint32_t d, m, p;
  GF_HD FastDiv() : d(1), m(0), p(0) {}
  GF_HD explicit FastDiv(uint32_t div) {
    d = div;
    uint32_t c = 0;
    while ((1ull << c) < div) c++;
    p = 31 + c;
    m = (uint32_t)(((1ull << p) + div - 1) / div);
  }
  GF_HD uint32_t div(uint32_t n) const { return (uint32_t)(((uint64_t)n * m) >> p); }
  GF_HD void divmod(uint32_t n, uint32_t &q, uint32_t &r) const {
    q = div(n);
    r = n - q * d;
  }
};

// Shared-memory padding: one spare element every 16 keeps the stride-R
// butterfly writes of the first Stockham stages free of bank conflicts for
// 8- and 16-byte elements.
GF_HD int spad(int i) { return i + (i >> 4); }
GF_HD int spad_size(int n) { return n + (n >> 4) + 1; }
