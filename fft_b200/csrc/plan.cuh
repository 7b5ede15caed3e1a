// plan.cuh -- host-side plan objects of the B200 FFT engine.
//
//   DevProg   one single-CTA line program (length n, precision): radix
//             schedule, threads per line, device twiddle planes.
//   Exec1D    a batched, strided 1-D complex transform of any length: one
//             fused launch (smooth lengths that fit one CTA, and Rader /
//             Bluestein whose convolution fits one CTA), a two-pass four-step
//             split, or a multi-pass convolution over a workspace.
//   ExecReal  the real forward/inverse of one length (packed half-length
//             transform for even n, full complex line for odd n).
//
// Routing follows the reference router (plan.go:42-73): powers of two and
// 13-smooth lengths are Cooley-Tukey, primes >= 700 are Rader (cyclic at
// p-1 when p-1 is 13-smooth, else padded-linear at bestConvLen(2(p-1))), and
// every other length is Bluestein at the next power of two >= 2n-1.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "dispatch.h"

namespace gf {

int set_err(int code, const std::string &msg);
const char *last_err();

inline size_t csize(int prec) { return prec == F64 ? 16 : 8; }
inline size_t rsize(int prec) { return prec == F64 ? 8 : 4; }
inline size_t twsize(int prec) { return prec == F32 ? 8 : 16; }
inline size_t spsize(int) { return 16; }

// integer routing helpers (plan.go, rader.go)
bool smooth13(long long n);
bool is_prime_ll(long long n);
long long primitive_root_ll(long long p);
bool conv_cost(long long m, double *cost);
long long best_conv_len(long long lo);
// Power-of-two part split into near-equal radices of at most 2^maxlog,
// then the odd primes.
std::vector<int> gpu_radices(long long n, int maxlog = 4);
void set_sched_variant(int prec, long long n, int v);
int get_sched_variant(int prec, long long n);
int sched_epoch();
// Caps the schedule variant for objects the calling thread builds while the
// guard lives.
struct SchedCap {
  int prev;
  explicit SchedCap(int cap);
  ~SchedCap();
};
// The tuning overrides as lists (for wisdom export) and a reset.
std::vector<std::array<long long, 3>> list_sched_variants();        // prec, n, variant
std::vector<std::array<long long, 5>> list_lpc_overrides();         // prec, n, op, colmode, lpc
std::vector<std::array<long long, 4>> list_pipe_overrides();        // prec, n, op, on
void clear_overrides();
void set_uneven_mode(int prec, int mode);  // 1 persistent, 0 per phase, -1 unset
int get_uneven_mode(int prec);

struct DevProg {
  int n = 0, prec = 0, maxe = 16, device = 0;
  int ctas = 1;  // in-shared-memory Rader: CTAs (a cluster) per signal
  LineProg lp{};
  void *tw = nullptr;
  void *tw_hi = nullptr;  // FP32-mixed: hi parts as FP32 pairs
  ~DevProg();
};

enum ExecKind { K_SINGLE = 0, K_FOURSTEP = 1, K_RADER = 2, K_BLUE = 3 };

struct DevProg;
// One line-kernel pass of a multi-pass transform.
struct RaderPhase {
  int op;
  std::shared_ptr<DevProg> prog;
  KArgs a;
  long long nlines;
};

struct Exec1D {
  long long n = 0;
  int prec = 0, kind = K_SINGLE, device = 0;
  std::shared_ptr<DevProg> prog;        // SINGLE: length n; fused conv: length cl / m
  std::shared_ptr<DevProg> p1, p2;      // FOURSTEP: lengths n1, n2
  std::shared_ptr<const Exec1D> sub;    // multi-pass convolution at cl / m
  long long n1 = 0, n2 = 0;
  void *tw4 = nullptr;                  // FOURSTEP: W_n^e for e < 2^tw4_sh, then W_n^(2^tw4_sh j)
  int tw4_sh = 0;                       //   (the split twiddle table of OpC2CTwiddle)
  bool fused = false;
  // Rader whose convolution fits one CTA's shared memory but not the
  // register-staged line kernels: the in-place kernel (rader_ip.cuh), with
  // its stage list in ipprog and the kernel spectrum in digit-reversed order
  bool inplace = false;
  std::shared_ptr<DevProg> ipprog;
  void *spec_ip = nullptr;
  long long cl = 0, g = 0, m = 0;
  int cyclic = 0;
  int *perm = nullptr, *iperm = nullptr;
  long long *jj = nullptr;
  void *spec = nullptr, *chirp = nullptr;
  ~Exec1D();
  size_t ws_bytes(long long nlines) const;
  int exec(const Side &in, const Side &out, long long nlines, int cj_in, int cj_out, double scale,
           void *ws, cudaStream_t st) const;
  int rader_two_pass(const Side &in, const Side &out, long long nlines, int cj_in, int cj_out, double scale,
                     void *ws, cudaStream_t st) const;
  void rader_phases(const Side &in, long long Din, const Side &out, long long Dout, long long nl, int cji,
                    int cjo, double scale, void *W1, void *W2, void *x0s, void *dc,
                    std::vector<RaderPhase> &ph) const;
  std::string describe() const;
};

enum RealMode { R_PACKED_FUSED = 0, R_PACKED_MULTI = 1, R_FULL_FUSED = 2, R_FULL_MULTI = 3 };

struct ExecReal {
  long long n = 0;
  int prec = 0, mode = R_FULL_FUSED, device = 0;
  std::shared_ptr<const Exec1D> cx;  // half (even) or full (odd) complex exec
  void *tw2 = nullptr;               // W_n^k, k = 0..n/2 (packed modes)
  void *tw2_hi = nullptr;            // FP32-mixed: hi parts as FP32 pairs
  ~ExecReal();
  size_t ws_bytes(long long nlines) const;
  // in: reals, out: bins.  wsc != 0 applies the real-spectrum edge-bin
  // weighting of the adjoints: bins 0 and n/2 times wsc, the others 2 wsc.
  // tiled_rows > 0: the bins side is the tiled intermediate of a rank-2
  // transform with that many rows per image (its Side's pointer is used,
  // nothing else); only packed fused plans (can_tile()) take it.
  int r2c(const Side &in, const Side &out, long long nlines, void *ws, cudaStream_t st,
          double wsc = 0.0, long long tiled_rows = 0) const;
  // in: bins (nb available per line), out: reals; the result is the
  // reference-normalised inverse (1/n) times `scale`.  halve: bins other than
  // 0 and n/2 enter halved (the adjoint of the forward's weighting).
  int c2r(const Side &in, int nb, const Side &out, long long nlines, double scale, void *ws,
          cudaStream_t st, bool halve = false, long long tiled_rows = 0) const;
  bool can_tile() const { return mode == R_PACKED_FUSED; }
  std::string describe() const;
};

// Cached constructors (per device, length, precision); nullptr + error set on
// failure.
std::shared_ptr<DevProg> get_prog(long long n, int prec);
std::shared_ptr<const Exec1D> get_exec(long long n, int prec);
std::shared_ptr<const ExecReal> get_real(long long n, int prec);
bool fits_single(long long n, int prec);
bool pairs_aligned(const Side &s, int prec);

bool side_simple(const Side &s, long long &D);
char *align256(char *p);
int choose_lpc(const DevProg &dp, const KArgs &a, int op, long long nlines, bool conv);
int choose_flags(int op, const KArgs &a);

// Calls the elementwise / table function `fn` of a precision's namespace
// (one counted launch).
#define GF_PREC_CALL(prec, fn, ...)                                                \
  (count_launch(), (prec) == F64 ? prec_f64::fn(__VA_ARGS__)                       \
                                 : ((prec) == F32 ? prec_f32::fn(__VA_ARGS__)      \
                                                  : prec_f32c::fn(__VA_ARGS__)))

// Launch helper for the line kernels.
int launch_line(int op, const DevProg &dp, KArgs a, long long nlines, cudaStream_t st,
                int lpc = 0, bool conv = false);

inline Side mk_side(void *p, long long dist_b, long long dist_l, long long stride, long long lpb) {
  Side s;
  s.ptr = p;
  s.dist_b = dist_b;
  s.dist_l = dist_l;
  s.stride = stride;
  s.lpb = FastDiv((uint32_t)(lpb < 1 ? 1 : lpb));
  s.boff = nullptr;
  return s;
}
// Contiguous lines of length len.
inline Side contig(void *p, long long len) { return mk_side(p, len, 0, 1, 1); }

// The TMA-fed persistent line kernel: on (default) or off for plain complex
// and packed real lines; pipe_status reads (and with clear, resets) the
// device's timeout word: 0, or 4 (timeout) with the error text set.
void set_tma_pipeline(int on);
int tma_pipeline();
void set_dependent_launch(int mode);
int dependent_launch();
int pipe_status(bool clear);

// Instrumentation (launch counter, CUDA-event timing per line kernel).
void count_launch();
long long launch_count();
void timing_enable(int on);
std::string timing_report();

// Autotuned lines-per-CTA overrides (key: prec, n, op, column-mode).
void set_lpc_override(int prec, long long n, int op, int colmode, int lpc);
int get_lpc_override(int prec, long long n, int op, int colmode);
void set_pipe_override(int prec, long long n, int op, int on);
int get_pipe_override(int prec, long long n, int op);

}  // namespace gf
