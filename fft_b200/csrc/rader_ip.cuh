// rader_ip.cuh -- Rader's prime-length transform with its whole convolution
// in one CTA's shared memory, for convolutions too long for the
// register-staged line kernels (e.g. p = 10007: cl = 20580 complex64, 165 KB).
//
// rader.go:129-172 restated for one signal per CTA:
//   a[k] = x[perm[k]] (k < q = p-1, zero to cl), A = FFT_cl(a),
//   X[0] = x0 + A[0], conv = IFFT_cl(A * B) = conj(FFT_cl(conj(A * B / cl))),
//   X[iperm[qi]] = x0 + conv[qi + off]   (off = 0 cyclic, q padded-linear).
// Both transforms run in place in shared memory, one butterfly per thread at
// a time (nothing register-staged, so the line needs no more registers than
// one radix-R butterfly):
//   forward  mixed-radix decimation in frequency, stages s = 0 .. nst-1: in
//            blocks of R_s * S_s elements, butterfly j < S_s takes
//            x[j + r S_s], runs DFT-R_s and multiplies output m by
//            W_{R_s S_s}^{j m}.  The spectrum comes out in digit-reversed
//            order: A[k] sits at pos(k) = sum_s m_s S_s for
//            k = m_0 + R_0 m_1 + R_0 R_1 m_2 + ...
//   product  the kernel spectrum B/cl is stored in the same digit-reversed
//            order, so the product is taken position by position
//   second   the transposed stages s = nst-1 .. 0 (twiddle the inputs, then
//            DFT-R_s): the transpose of the forward factorisation is again a
//            forward DFT (the DFT matrix is symmetric), and it reads
//            digit-reversed input and writes natural order.
// KArgs: lp holds the stage list (radix[s] = R_s, ns[s] = S_s, twoff[s],
// nsdiv[s] divides by S_s, tw the twiddle planes W_{R S}^{j m} in the
// precision's twiddle form); aux0 = perm, aux1 = iperm (int32, q each),
// aux2 = B/cl in digit-reversed order (sp_t), ia = p, ic = off.
#pragma once
#include "ops.cuh"

namespace gf {

template <class P, int R>
GF_DEV void rip_dif_stage(typename P::cpx *x, int cl, int S, FastDiv sd, const typename P::tw_t *tw) {
  using C = typename P::cpx;
  const int nb = cl / R;
  for (int bi = threadIdx.x; bi < nb; bi += blockDim.x) {
    uint32_t blk, j;
    sd.divmod((uint32_t)bi, blk, j);
    C *p = x + (size_t)blk * (R * S) + j;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = p[r * S];
    Dft<R, C>::run(v);
    if (S > 1) {
#pragma unroll
      for (int m = 1; m < R; m++) v[m] = twmul(v[m], ld_keep(&tw[(m - 1) * S + j]));
    }
#pragma unroll
    for (int m = 0; m < R; m++) p[m * S] = v[m];
  }
}

template <class P, int R>
GF_DEV void rip_dit_stage(typename P::cpx *x, int cl, int S, FastDiv sd, const typename P::tw_t *tw) {
  using C = typename P::cpx;
  const int nb = cl / R;
  for (int bi = threadIdx.x; bi < nb; bi += blockDim.x) {
    uint32_t blk, j;
    sd.divmod((uint32_t)bi, blk, j);
    C *p = x + (size_t)blk * (R * S) + j;
    C v[R];
#pragma unroll
    for (int m = 0; m < R; m++) v[m] = p[m * S];
    if (S > 1) {
#pragma unroll
      for (int m = 1; m < R; m++) v[m] = twmul(v[m], ld_keep(&tw[(m - 1) * S + j]));
    }
    Dft<R, C>::run(v);
#pragma unroll
    for (int r = 0; r < R; r++) p[r * S] = v[r];
  }
}

// Radices a convolution length may use here (prime factors up to 13, powers
// of two split into stages of at most 8).
GF_HD bool rip_radix_ok(int R) {
  return R == 2 || R == 3 || R == 4 || R == 5 || R == 7 || R == 8 || R == 11 || R == 13;
}

template <class P>
GF_DEV void rip_stage(bool dit, int R, typename P::cpx *x, int cl, int S, FastDiv sd, const typename P::tw_t *tw) {
#define GF_RIP_CASE(RR)                                    \
  case RR:                                                 \
    if (dit) rip_dit_stage<P, RR>(x, cl, S, sd, tw);       \
    else rip_dif_stage<P, RR>(x, cl, S, sd, tw);           \
    break;
  switch (R) {
    GF_RIP_CASE(2)
    GF_RIP_CASE(3)
    GF_RIP_CASE(4)
    GF_RIP_CASE(5)
    GF_RIP_CASE(7)
    GF_RIP_CASE(8)
    GF_RIP_CASE(11)
    GF_RIP_CASE(13)
    default: break;
  }
#undef GF_RIP_CASE
}

// One signal (`line` of the launch) on all the CTA's threads, in the
// dynamic shared memory (cl complex values).
template <class P> GF_DEV void rader_ip_line(const KArgs &a, long long line) {
  using C = typename P::cpx;
  using Rl = typename P::real;
  using TW = typename P::tw_t;
  using SP = typename P::sp_t;
  C *x = smem_base<C>();
  __shared__ C s_x0, s_X0;
  const LineProg &lp = a.lp;
  const int cl = lp.n, p = (int)a.ia, q = p - 1, off = a.ic;
  const int *perm = (const int *)a.aux0;
  const int *iperm = (const int *)a.aux1;
  const SP *B = (const SP *)a.aux2;
  const TW *tw = (const TW *)lp.tw;
  const C *in = (const C *)a.in.ptr + line_off(a.in, (uint32_t)line);
  const long long ist = a.in.stride;
  for (int k = threadIdx.x; k < cl; k += blockDim.x) {
    C v = mkc((Rl)0, (Rl)0);
    if (k < q) {
      v = in[(long long)__ldg(&perm[k]) * ist];
      if (a.cj_in) v.y = -v.y;
    }
    x[k] = v;
  }
  if (threadIdx.x == 0) {
    C v = in[0];
    if (a.cj_in) v.y = -v.y;
    s_x0 = v;
  }
  __syncthreads();
  for (int s = 0; s < lp.nst; s++) {
    rip_stage<P>(false, lp.radix[s], x, cl, lp.ns[s], lp.nsdiv[s], tw + lp.twoff[s]);
    __syncthreads();
  }
  // X[0] = x0 + A[0] (A[0] sits at position 0), then conj(A * B / cl)
  if (threadIdx.x == 0) s_X0 = cadd(s_x0, x[0]);
  __syncthreads();
  for (int k = threadIdx.x; k < cl; k += blockDim.x) x[k] = cconj(spmul(x[k], __ldg(&B[k])));
  __syncthreads();
  for (int s = lp.nst - 1; s >= 0; s--) {
    rip_stage<P>(true, lp.radix[s], x, cl, lp.ns[s], lp.nsdiv[s], tw + lp.twoff[s]);
    __syncthreads();
  }
  C *out = (C *)a.out.ptr + line_off(a.out, (uint32_t)line);
  const long long ost = a.out.stride;
  const Rl sc = (Rl)a.scale;
  const Rl sy = a.cj_out ? -sc : sc;
  for (int i = threadIdx.x; i < p; i += blockDim.x) {
    C y;
    long long d;
    if (i == 0) {
      y = s_X0;
      d = 0;
    } else {
      y = cadd(s_x0, cconj(x[i - 1 + off]));
      d = __ldg(&iperm[i - 1]);
    }
    out[d * ost] = mkc(y.x * sc, y.y * sy);
  }
  __syncthreads();  // the next signal overwrites x and s_x0
}

// Threads per CTA: 1024 for complex64 (64 registers hold any butterfly up to
// radix 13), 512 for complex128 (twice the registers per element).
template <class P> constexpr int rip_threads() { return sizeof(typename P::cpx) == 16 ? 512 : 1024; }

// One CTA per signal at a time (persistent over the launch's signals).
template <class P>
__global__ void __launch_bounds__(rip_threads<P>(), 1) k_rader_ip(const KArgs a) {
  for (long long line = blockIdx.x; line < a.nlines; line += gridDim.x) rader_ip_line<P>(a, line);
}

// ---------------------------------------------------------------------------
// Two-CTA form, for convolutions up to twice one CTA's shared memory (FP64
// p = 10007: cl = 20580 complex128, 329 KB).  The two CTAs of a cluster
// share one signal: CTA c holds positions [c H, (c+1) H), H = cl / 2.  With
// an even first radix R_0, stage 0's blocks are the whole line but every
// later stage's blocks (S_0 = cl / R_0 elements at most, H a multiple of S_0)
// lie inside one half, and so does the position-by-position product.  Only
// stage 0 of the forward transform and the last transposed stage of the
// second one read and write the partner's half, through distributed shared
// memory (plain loads and stores to the partner CTA's shared window, no bulk
// copies), each between two cluster barriers.
// ---------------------------------------------------------------------------

// Stage 0 on the pair: butterfly j (j < S) takes positions j + r S, r < R;
// r < R/2 lie in CTA 0's half at offset j + r S, the others in CTA 1's at
// j + (r - R/2) S.  CTA `rank` takes the butterflies j in its share of [0, S).
template <class P, int R>
GF_DEV void rip2_stage0(bool dit, typename P::cpx *h0, typename P::cpx *h1, int S, const typename P::tw_t *tw,
                        unsigned rank) {
  using C = typename P::cpx;
  constexpr int RH = R / 2;
  const int jm = (S + 1) / 2;
  const int j0 = rank ? jm : 0, j1 = rank ? S : jm;
  for (int j = j0 + (int)threadIdx.x; j < j1; j += blockDim.x) {
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = (r < RH ? h0 : h1)[j + (r % RH) * S];
    if (dit) {
#pragma unroll
      for (int m = 1; m < R; m++) v[m] = twmul(v[m], ld_keep(&tw[(m - 1) * S + j]));
      Dft<R, C>::run(v);
    } else {
      Dft<R, C>::run(v);
#pragma unroll
      for (int m = 1; m < R; m++) v[m] = twmul(v[m], ld_keep(&tw[(m - 1) * S + j]));
    }
#pragma unroll
    for (int r = 0; r < R; r++) (r < RH ? h0 : h1)[j + (r % RH) * S] = v[r];
  }
}

template <class P>
GF_DEV void rip2_stage0_any(bool dit, int R, typename P::cpx *h0, typename P::cpx *h1, int S,
                            const typename P::tw_t *tw, unsigned rank) {
  switch (R) {
    case 2: rip2_stage0<P, 2>(dit, h0, h1, S, tw, rank); break;
    case 4: rip2_stage0<P, 4>(dit, h0, h1, S, tw, rank); break;
    case 8: rip2_stage0<P, 8>(dit, h0, h1, S, tw, rank); break;
    default: break;
  }
}

// Whether a stage list suits the pair: an even first radix with a shared-
// memory butterfly (the host puts the power-of-two radices first).
GF_HD bool rip2_first_radix_ok(int R) { return R == 2 || R == 4 || R == 8; }

GF_DEV unsigned rip2_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// Barrier over both CTAs of the cluster; release/acquire order each CTA's
// shared-memory writes (its own half and the partner's) before the
// partner's reads that follow.
GF_DEV void rip2_cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Generic address of the same shared-memory location in CTA `rank` of the
// cluster.
template <class T> GF_DEV T *rip2_map(T *p, unsigned rank) {
  uint64_t d;
  asm volatile("mapa.u64 %0, %1, %2;" : "=l"(d) : "l"(reinterpret_cast<uint64_t>(p)), "r"(rank));
  return reinterpret_cast<T *>(d);
}

template <class P> GF_DEV void rader_ip2_line(const KArgs &a, long long line, unsigned rank) {
  using C = typename P::cpx;
  using Rl = typename P::real;
  using TW = typename P::tw_t;
  using SP = typename P::sp_t;
  C *x = smem_base<C>();
  __shared__ C s_x0, s_X0;
  const LineProg &lp = a.lp;
  const int cl = lp.n, H = cl / 2, base = (int)rank * H, p = (int)a.ia, q = p - 1, off = a.ic;
  const int *perm = (const int *)a.aux0;
  const int *iperm = (const int *)a.aux1;
  const SP *B = (const SP *)a.aux2 + base;
  const TW *tw = (const TW *)lp.tw;
  C *h0 = rip2_map(x, 0), *h1 = rip2_map(x, 1);
  const C *in = (const C *)a.in.ptr + line_off(a.in, (uint32_t)line);
  const long long ist = a.in.stride;
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    C v = mkc((Rl)0, (Rl)0);
    if (base + k < q) {
      v = in[(long long)__ldg(&perm[base + k]) * ist];
      if (a.cj_in) v.y = -v.y;
    }
    x[k] = v;
  }
  if (threadIdx.x == 0) {
    C v = in[0];
    if (a.cj_in) v.y = -v.y;
    s_x0 = v;
  }
  rip2_cluster_sync();  // both halves gathered
  rip2_stage0_any<P>(false, lp.radix[0], h0, h1, lp.ns[0], tw + lp.twoff[0], rank);
  rip2_cluster_sync();  // stage 0's writes to either half visible to its owner
  for (int s = 1; s < lp.nst; s++) {
    rip_stage<P>(false, lp.radix[s], x, H, lp.ns[s], lp.nsdiv[s], tw + lp.twoff[s]);
    __syncthreads();
  }
  // X[0] = x0 + A[0] (position 0, in CTA 0), then conj(A * B / cl)
  if (rank == 0 && threadIdx.x == 0) s_X0 = cadd(s_x0, x[0]);
  __syncthreads();
  for (int k = threadIdx.x; k < H; k += blockDim.x) x[k] = cconj(spmul(x[k], __ldg(&B[k])));
  __syncthreads();
  for (int s = lp.nst - 1; s >= 1; s--) {
    rip_stage<P>(true, lp.radix[s], x, H, lp.ns[s], lp.nsdiv[s], tw + lp.twoff[s]);
    __syncthreads();
  }
  rip2_cluster_sync();  // both halves through the local stages
  rip2_stage0_any<P>(true, lp.radix[0], h0, h1, lp.ns[0], tw + lp.twoff[0], rank);
  rip2_cluster_sync();  // the transposed stage 0 complete in both halves; no
                        // remote access until the next signal's first barrier
  C *out = (C *)a.out.ptr + line_off(a.out, (uint32_t)line);
  const long long ost = a.out.stride;
  const Rl sc = (Rl)a.scale;
  const Rl sy = a.cj_out ? -sc : sc;
  // output i >= 1 reads position i - 1 + off: this CTA writes the outputs
  // whose position lies in its half, CTA 0 also X[0]
  const int i0 = base - off + 1 > 1 ? base - off + 1 : 1, i1 = base + H - off + 1 < p ? base + H - off + 1 : p;
  if (rank == 0 && threadIdx.x == 0) out[0] = mkc(s_X0.x * sc, s_X0.y * sy);
  for (int i = i0 + (int)threadIdx.x; i < i1; i += blockDim.x) {
    const C y = cadd(s_x0, cconj(x[i - 1 + off - base]));
    out[(long long)__ldg(&iperm[i - 1]) * ost] = mkc(y.x * sc, y.y * sy);
  }
  __syncthreads();  // the next signal overwrites x and s_x0
}

// One cluster of two CTAs per signal at a time (persistent over the signals:
// both CTAs of a cluster take the same signals, so they meet the same
// cluster barriers).
template <class P>
__global__ void __launch_bounds__(rip_threads<P>(), 1) k_rader_ip2(const KArgs a) {
  const unsigned rank = rip2_rank();
  const long long ncl = gridDim.x / 2;
  for (long long line = blockIdx.x / 2; line < a.nlines; line += ncl) rader_ip2_line<P>(a, line, rank);
}

}  // namespace gf
