// tables.cu -- integer and chirp tables built on the device at plan time.
#include "dispatch.h"
#include "kernels.cuh"

namespace gf {

// Rader permutations (rader.go:67-72): perm[k] = g^k mod p, iperm[qi] =
// perm[(q - qi) mod q]; both bit-exact integer work.
GF_DEV long long modpow_dev(long long b, long long e, long long m) {
  long long r = 1;
  b %= m;
  while (e > 0) {
    if (e & 1) r = r * b % m;
    e >>= 1;
    b = b * b % m;
  }
  return r;
}
__global__ void k_gen_rader_perm(int *perm, int *iperm, long long p, long long g) {
  const long long q = p - 1;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < q;
       k += (long long)gridDim.x * blockDim.x) {
    perm[k] = (int)modpow_dev(g, k, p);
    iperm[k] = (int)modpow_dev(g, (q - k) % q, p);
  }
}
// Rader convolution kernel b (rader.go:101-125): for m < q (cyclic) or m < 2q
// (padded linear), b[m] = W_p^{perm[(q - (m mod q)) mod q]}; zero elsewhere.
// Written in FP64 as the input of an FP64 FFT.
__global__ void k_gen_rader_kernel(double2 *b, const int *perm, long long p, long long cl,
                                   int cyclic) {
  const long long q = p - 1;
  const long long lim = cyclic ? q : 2 * q;
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < cl;
       m += (long long)gridDim.x * blockDim.x) {
    if (m < lim) {
      const long long s = m % q;
      b[m] = root_of_unity(perm[(q - s) % q], p);
    } else {
      b[m] = make_double2(0.0, 0.0);
    }
  }
}
// Bluestein chirp index jj = j*j mod 2n (bluestein.go:38), bit-exact in 64-bit
// integers, and the forward chirp w[j] = exp(-pi i jj / n) = W_{2n}^{jj}.
__global__ void k_gen_chirp(long long *jj, double2 *w, long long n) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const long long e = (j * j) % (2 * n);
    jj[j] = e;
    w[j] = root_of_unity(e, 2 * n);
  }
}
// Bluestein kernel (bluestein.go:52-63): b[0] = conj w[0], b[j] = b[m-j] =
// conj w[j] for 0 < j < n, zero elsewhere.
__global__ void k_gen_blue_kernel(double2 *b, const double2 *w, long long n, long long m) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m;
       k += (long long)gridDim.x * blockDim.x) {
    double2 v = make_double2(0.0, 0.0);
    if (k < n) v = make_double2(w[k].x, -w[k].y);
    else if (m - k < n) v = make_double2(w[m - k].x, -w[m - k].y);
    b[k] = v;
  }
}

static unsigned tb_blocks(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

cudaError_t gen_rader_perm(int *perm, int *iperm, long long p, long long g, cudaStream_t st) {
  k_gen_rader_perm<<<tb_blocks(p), 256, 0, st>>>(perm, iperm, p, g);
  return cudaGetLastError();
}
cudaError_t gen_rader_kernel(double2 *b, const int *perm, long long p, long long cl, int cyclic,
                             cudaStream_t st) {
  k_gen_rader_kernel<<<tb_blocks(cl), 256, 0, st>>>(b, perm, p, cl, cyclic);
  return cudaGetLastError();
}
cudaError_t gen_chirp(long long *jj, double2 *w, long long n, cudaStream_t st) {
  k_gen_chirp<<<tb_blocks(n), 256, 0, st>>>(jj, w, n);
  return cudaGetLastError();
}
cudaError_t gen_blue_kernel(double2 *b, const double2 *w, long long n, long long m, cudaStream_t st) {
  k_gen_blue_kernel<<<tb_blocks(m), 256, 0, st>>>(b, w, n, m);
  return cudaGetLastError();
}

// Symmetric windows (window.go:20-100) in FP64 on the device, stored in the
// output's precision.  Cosine windows w[k] = sum_j (-1)^j a_j cos(2 pi j k /
// (n-1)) take each angle from the exact integer residue j k mod (n-1), so
// cospi's argument is reduced without rounding; Bartlett is the triangle
// (2/(n-1)) ((n-1)/2 - |k - (n-1)/2|).  kind: 0 Hann, 1 Hamming, 2 Blackman,
// 3 Blackman-Harris, 4 Bartlett.
template <class R>
__global__ void k_gen_window(R *w, long long n, int kind) {
  const double a[4][4] = {{0.5, 0.5, 0, 0}, {0.54, 0.46, 0, 0}, {0.42, 0.5, 0.08, 0},
                          {0.35875, 0.48829, 0.14128, 0.01168}};
  const int na = kind == 2 ? 3 : (kind == 3 ? 4 : 2);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    double v;
    if (n == 1) {
      v = 1.0;
    } else if (kind == 4) {
      const double denom = (double)(n - 1), half = denom / 2;
      v = (2 / denom) * (half - fabs((double)k - half));
    } else {
      v = a[kind][0];
      double sign = -1.0;
      for (int j = 1; j < na; j++) {
        const long long e = ((long long)j * k) % (n - 1);
        v += sign * a[kind][j] * cospi(2.0 * (double)e / (double)(n - 1));
        sign = -sign;
      }
    }
    w[k] = (R)v;
  }
}

cudaError_t gen_window(void *w, int prec_bytes, long long n, int kind, cudaStream_t st) {
  if (prec_bytes == 8)
    k_gen_window<double><<<tb_blocks(n), 256, 0, st>>>((double *)w, n, kind);
  else
    k_gen_window<float><<<tb_blocks(n), 256, 0, st>>>((float *)w, n, kind);
  return cudaGetLastError();
}

}  // namespace gf
