// plan.cu -- line programs, 1-D executors and real executors.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <sstream>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "pipe.h"
#include "pipe.cuh"
#include "plan.cuh"
#include "rader_ip.cuh"

namespace gf {

static thread_local std::string g_err;
int set_err(int code, const std::string &msg) {
  g_err = msg;
  return code;
}
const char *last_err() { return g_err.c_str(); }

#define GF_CK(x)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess)                                                              \
      return set_err(3, std::string(#x) + ": " + cudaGetErrorString(e_));               \
  } while (0)

// ---------------------------------------------------------------------------
// Integer helpers, restated from the reference router.
// ---------------------------------------------------------------------------

// plan.go:134-141
bool smooth13(long long n) {
  if (n < 1) return false;
  for (long long p : {2, 3, 5, 7, 11, 13})
    while (n % p == 0) n /= p;
  return n == 1;
}

// rader.go:232-245
bool is_prime_ll(long long n) {
  if (n < 2) return false;
  if (n % 2 == 0) return n == 2;
  for (long long d = 3; d * d <= n; d += 2)
    if (n % d == 0) return false;
  return true;
}

static long long modpow_h(long long b, long long e, long long m) {
  long long r = 1;
  b %= m;
  while (e > 0) {
    if (e & 1) r = (__int128)r * b % m;
    e >>= 1;
    b = (__int128)b * b % m;
  }
  return r;
}

// rader.go:178-212: smallest generator of (Z/pZ)*.
long long primitive_root_ll(long long p) {
  long long phi = p - 1, m = phi;
  std::vector<long long> f;
  for (long long d = 2; d * d <= m; d++)
    if (m % d == 0) {
      f.push_back(d);
      while (m % d == 0) m /= d;
    }
  if (m > 1) f.push_back(m);
  if (f.empty()) return 1;
  for (long long g = 2;; g++) {
    bool gen = true;
    for (long long q : f)
      if (modpow_h(g, phi / q, p) == 1) {
        gen = false;
        break;
      }
    if (gen) return g;
  }
}

// plan.go:192-220
bool conv_cost(long long m, double *cost) {
  const double w2 = 2.0, w3 = 2.0, w5 = 2.8, w7 = 2.6;
  double c = 0;
  long long x = m;
  while (x % 4 == 0) { c += w2; x /= 4; }
  while (x % 2 == 0) { c += w2; x /= 2; }
  while (x % 3 == 0) { c += w3; x /= 3; }
  while (x % 5 == 0) { c += w5; x /= 5; }
  while (x % 7 == 0) { c += w7; x /= 7; }
  if (x != 1) return false;
  if (cost) *cost = (double)m * c;
  return true;
}

// plan.go:241-259
long long best_conv_len(long long lo) {
  if (lo < 1) lo = 1;
  long long hi = lo + (lo * 4 + 9) / 10, best = lo;
  double bc = 0;
  bool have = false;
  for (long long m = lo; m <= hi; m++) {
    double c;
    if (!conv_cost(m, &c)) continue;
    if (!have || c < bc) { best = m; bc = c; have = true; }
  }
  return best;
}

// Schedule variants per (precision, length): 0 = radices up to 16 with 16
// (FP64) or up to 32 (FP32) elements per thread; 1 = radices up to 8 with 8
// elements per thread (twice the threads per line, about half the registers,
// more resident warps, one more stage); 2 (FP32 forms) = radices up to 32
// with 32 elements per thread (fewer stages: fewer barriers, shared-memory
// exchanges and twiddle loads, more registers).  Objects built under one setting are
// cached apart from those built under another (the epoch is part of every
// cache key).
static std::mutex g_sched_mu;
static std::map<std::pair<int, long long>, int> g_sched;
static std::atomic<int> g_sched_epoch{0};
void set_sched_variant(int prec, long long n, int v) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  if (v <= 0) g_sched.erase(std::make_pair(prec, n));
  else g_sched[std::make_pair(prec, n)] = v;
  g_sched_epoch.fetch_add(1);
}
// Highest variant the calling thread may build (uneven batches run every
// line in one persistent kernel with 16-element registers, so they cap at 1).
static thread_local int t_sched_cap = 2;
SchedCap::SchedCap(int cap) : prev(t_sched_cap) { t_sched_cap = cap; }
SchedCap::~SchedCap() { t_sched_cap = prev; }
int get_sched_variant(int prec, long long n) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  auto it = g_sched.find(std::make_pair(prec, n));
  const int v = it == g_sched.end() ? 0 : it->second;
  return std::min(v, t_sched_cap);
}
// Cache-key part of the settings: the override epoch and the thread's cap.
int sched_epoch() { return g_sched_epoch.load() * 4 + t_sched_cap; }
// Uneven-batch execution per precision: persistent kernel (1) or one launch
// per phase (0); -1 = not set (persistent).
static std::atomic<int> g_uneven_mode[3] = {{-1}, {-1}, {-1}};
void set_uneven_mode(int prec, int mode) {
  if (prec >= 0 && prec < 3) g_uneven_mode[prec].store(mode);
}
int get_uneven_mode(int prec) { return (prec >= 0 && prec < 3) ? g_uneven_mode[prec].load() : -1; }
std::vector<std::array<long long, 3>> list_sched_variants() {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  std::vector<std::array<long long, 3>> v;
  for (auto &kv : g_sched) v.push_back({kv.first.first, kv.first.second, kv.second});
  return v;
}

// Radix schedule of a 13-smooth length for the Stockham stages: the power of
// two is split into as few stages of radix at most 2^maxlog as possible with
// the bits spread evenly, then one stage per odd prime factor.
std::vector<int> gpu_radices(long long n, int maxlog) {
  std::vector<int> r;
  long long m = n;
  int a = 0;
  while (m % 2 == 0) { a++; m /= 2; }
  if (a > 0) {
    int k = (a + maxlog - 1) / maxlog;
    for (int i = 0; i < k; i++) r.push_back(1 << (a / k + (i < a % k ? 1 : 0)));
  }
  for (int p : {3, 5, 7, 11, 13})
    while (m % p == 0) { r.push_back(p); m /= p; }
  return r;
}

// ---------------------------------------------------------------------------
// Device properties and kernel lookup.
// ---------------------------------------------------------------------------
static int cur_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

static size_t max_smem_optin() {
  static std::mutex mu;
  static std::map<int, size_t> cache;
  int d = cur_device();
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(d);
  if (it != cache.end()) return it->second;
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, d) != cudaSuccess || v <= 0)
    v = 48 * 1024;
  cache[d] = (size_t)v;
  return (size_t)v;
}

static KFn kernel_for(int prec, int maxe, int op) {
  const bool g0 = op == OP_C2C || op == OP_C2C_TW || op == OP_RADER || op == OP_BLUE || op == OP_RADER_FS1 ||
                  op == OP_RADER_FS2 || op == OP_RADER_FS4 || op == OP_FILTER_COL;
  switch (prec) {
    case F64: return g0 ? line_kernel_f64_0(maxe, op) : line_kernel_f64_1(maxe, op);
    case F32: return g0 ? line_kernel_f32_0(maxe, op) : line_kernel_f32_1(maxe, op);
    default: return g0 ? line_kernel_f32c_0(maxe, op) : line_kernel_f32c_1(maxe, op);
  }
}

static KFn kernel_ct_for(const DevProg &dp, int op, int lpc, bool pipe) {
  const bool g0 = op == OP_C2C || op == OP_C2C_TW || op == OP_FILTER_COL;
  const int n = dp.n, T = dp.lp.T, nst = dp.lp.nst;
  const int *r = dp.lp.radix;
  switch (dp.prec) {
    case F64:
      return g0 ? line_kernel_ct_f64_0(n, T, lpc, op, r, nst, pipe) : line_kernel_ct_f64_1(n, T, lpc, op, r, nst, pipe);
    case F32:
      return g0 ? line_kernel_ct_f32_0(n, T, lpc, op, r, nst, pipe) : line_kernel_ct_f32_1(n, T, lpc, op, r, nst, pipe);
    default:
      return g0 ? line_kernel_ct_f32c_0(n, T, lpc, op, r, nst, pipe)
                : line_kernel_ct_f32c_1(n, T, lpc, op, r, nst, pipe);
  }
}

static int num_sms() {
  static int v = 0;
  if (!v) {
    int d = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
    if (v <= 0) v = 148;
  }
  return v;
}

static int ensure_smem(KFn f, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> done;
  if (smem <= 48 * 1024) return 0;
  auto key = std::make_pair(cur_device(), (const void *)f);
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find(key);
  if (it != done.end() && it->second >= smem) return 0;
  GF_CK(cudaFuncSetAttribute((const void *)f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  done[key] = smem;
  return 0;
}

// ---------------------------------------------------------------------------
// DevProg
// ---------------------------------------------------------------------------
DevProg::~DevProg() {
  if (tw) cudaFree(tw);
  if (tw_hi) cudaFree(tw_hi);
}

static int pick_threads(long long n, int maxe, const std::vector<int> &rad) {
  long long T = (n + maxe - 1) / maxe;
  if (T < 1) T = 1;
  for (; T <= 512; T++) {
    bool ok = true;
    for (int R : rad) {
      const long long nb = n / R, per = (nb + T - 1) / T;
      if (per > maxe / R) { ok = false; break; }
    }
    if (ok) return (int)T;
  }
  return -1;
}

static bool schedule_for(long long n, int prec, int &maxe, int &T, std::vector<int> &rad) {
  if (n < 1 || !smooth13(n)) return false;
  const size_t bytes = (size_t)spad_size((int)n) * csize(prec) + 2 * csize(prec);
  if (bytes > max_smem_optin()) return false;
  const int var = get_sched_variant(prec, n);
  if (var == 1) {
    rad = gpu_radices(n, 3);
    const int t = (int)rad.size() <= GF_MAXST ? pick_threads(n, 8, rad) : -1;
    if (t > 0) {
      maxe = 8;
      T = t;
      return true;
    }
  }
  if (var == 2 && prec != F64) {
    rad = gpu_radices(n, 5);
    const int t = (int)rad.size() <= GF_MAXST ? pick_threads(n, 32, rad) : -1;
    if (t > 0) {
      maxe = 32;
      T = t;
      return true;
    }
  }
  rad = gpu_radices(n, 4);
  if ((int)rad.size() > GF_MAXST) return false;
  for (int me : {16, 32}) {
    if (me == 32 && prec == F64) break;
    const int t = pick_threads(n, me, rad);
    if (t > 0) {
      maxe = me;
      T = t;
      return true;
    }
  }
  return false;
}

bool fits_single(long long n, int prec) {
  int me, T;
  std::vector<int> rad;
  if (n <= 1) return true;
  return schedule_for(n, prec, me, T, rad);
}

static int build_prog(long long n, int prec, std::shared_ptr<DevProg> &out) {
  auto dp = std::make_shared<DevProg>();
  dp->n = (int)n;
  dp->prec = prec;
  dp->device = cur_device();
  LineProg &lp = dp->lp;
  lp.n = (int)n;
  if (n <= 1) {
    lp.nst = 0;
    lp.T = 1;
    lp.maxe = 16;
    dp->maxe = 16;
    out = dp;
    return 0;
  }
  int maxe = 16, T = 1;
  std::vector<int> rad;
  if (!schedule_for(n, prec, maxe, T, rad))
    return set_err(5, "length " + std::to_string(n) + " has no single-CTA schedule");
  lp.nst = (int)rad.size();
  lp.T = T;
  lp.maxe = maxe;
  dp->maxe = maxe;
  StageTab tab{};
  tab.nst = lp.nst;
  long long ns = 1, off = 0;
  for (int s = 0; s < lp.nst; s++) {
    lp.radix[s] = tab.radix[s] = rad[s];
    lp.ns[s] = tab.ns[s] = (int)ns;
    lp.twoff[s] = tab.twoff[s] = (int)off;
    lp.nsdiv[s] = FastDiv((uint32_t)ns);
    off += ns * (rad[s] - 1);
    ns *= rad[s];
  }
  const long long total = off > 0 ? off : 1;
  GF_CK(cudaMalloc(&dp->tw, total * twsize(prec)));
  lp.tw = dp->tw;
  cudaError_t e = cudaSuccess;
  switch (prec) {
    case F64: e = prec_f64::stage_tw(dp->tw, tab, off, 0); break;
    case F32: e = prec_f32::stage_tw(dp->tw, tab, off, 0); break;
    default: e = prec_f32c::stage_tw(dp->tw, tab, off, 0); break;
  }
  GF_CK(e);
  if (prec == F32C) {
    // the hi parts as a compact FP32 table, for the short-line kernels
    GF_CK(cudaMalloc(&dp->tw_hi, total * twsize(F32)));
    lp.tw_hi = dp->tw_hi;
    GF_CK(prec_f32::stage_tw(dp->tw_hi, tab, off, 0));
  }
  GF_CK(cudaStreamSynchronize(0));
  out = dp;
  return 0;
}

template <class K, class V>
static std::shared_ptr<V> cache_get(std::map<K, std::shared_ptr<V>> &c, std::mutex &mu, const K &k) {
  std::lock_guard<std::mutex> lk(mu);
  auto it = c.find(k);
  return it == c.end() ? nullptr : it->second;
}

std::shared_ptr<DevProg> get_prog(long long n, int prec) {
  static std::mutex mu;
  static std::map<std::tuple<int, long long, int, int>, std::shared_ptr<DevProg>> cache;
  auto key = std::make_tuple(cur_device(), n, prec, sched_epoch());
  if (auto p = cache_get(cache, mu, key)) return p;
  std::shared_ptr<DevProg> p;
  if (build_prog(n, prec, p) != 0) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;  // another thread won the race
  cache[key] = p;
  return p;
}

// ---------------------------------------------------------------------------
// Instrumentation: a launch counter and optional CUDA-event timing of every
// line-kernel launch (events recorded on the launch stream around it).
// ---------------------------------------------------------------------------
static std::atomic<long long> g_launches{0};
static std::atomic<int> g_timing{0};
struct TimingRec {
  std::string key;
  cudaEvent_t a, b;
  double bytes;
};
static std::mutex g_tmu;
static std::vector<TimingRec> g_trecs;

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(); }
void timing_enable(int on) { g_timing.store(on ? 1 : 0); }

std::string timing_report() {
  std::vector<TimingRec> recs;
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    recs.swap(g_trecs);
  }
  struct Agg { long long launches = 0; double ms = 0, bytes = 0; };
  std::map<std::string, Agg> agg;
  for (auto &r : recs) {
    float ms = 0;
    cudaEventSynchronize(r.b);
    cudaEventElapsedTime(&ms, r.a, r.b);
    Agg &g = agg[r.key];
    g.launches++;
    g.ms += ms;
    g.bytes += r.bytes;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  std::ostringstream o;
  o << "[";
  bool first = true;
  for (auto &kv : agg) {
    o << (first ? "" : ",") << "{\"kernel\":\"" << kv.first << "\",\"launches\":" << kv.second.launches
      << ",\"ms\":" << kv.second.ms << ",\"bytes\":" << kv.second.bytes << "}";
    first = false;
  }
  o << "]";
  return o.str();
}

static const char *op_name(int op) {
  static const char *n[] = {"c2c", "c2c_twiddle", "r2c_packed", "c2r_packed", "r2c_full", "c2r_full",
                            "rader_fused", "bluestein_fused", "spectrogram", "rader_fs1", "rader_fs2",
                            "rader_fs4", "filter_col", "rader_inplace"};
  return (op >= 0 && op < OP_COUNT) ? n[op] : "?";
}

// Compulsory bytes (input + output) of one launch.
static double algo_bytes(int op, const DevProg &dp, const KArgs &a, long long nl) {
  const double c = (double)csize(dp.prec), r = (double)rsize(dp.prec), n = dp.n;
  switch (op) {
    case OP_R2C:
    case OP_C2R: return nl * (2 * n * r + (n + 1) * c);
    case OP_R2C_FULL:
    case OP_C2R_FULL: return nl * (n * r + (double)(dp.n / 2 + 1) * c);
    case OP_RADER:
    case OP_RADER_IP:
    case OP_BLUE: return 2.0 * nl * (double)a.ia * c;
    case OP_SPECTRO: return nl * (2 * n * r + (n + 1) * r);
    case OP_FILTER_COL: {
      // spectrum in and out, H read; X saved (forward) or X read and the
      // per-image dH term written (adjoint)
      const int extra = ((a.ic & GF_FILT_SAVE) ? 1 : 0) + ((a.ic & GF_FILT_DH) ? 2 : 0);
      return nl * n * c * (3.0 + extra);
    }
    default: return 2.0 * nl * n * c;
  }
}

// ---------------------------------------------------------------------------
// Launch
// ---------------------------------------------------------------------------
static std::mutex g_lpc_mu;
static std::map<std::tuple<int, long long, int, int>, int> g_lpc;
static std::map<std::tuple<int, long long, int>, int> g_pipe;
void set_pipe_override(int prec, long long n, int op, int on) {
  std::lock_guard<std::mutex> lk(g_lpc_mu);
  g_pipe[std::make_tuple(prec, n, op)] = on;
}
int get_pipe_override(int prec, long long n, int op) {
  std::lock_guard<std::mutex> lk(g_lpc_mu);
  auto it = g_pipe.find(std::make_tuple(prec, n, op));
  return it == g_pipe.end() ? 0 : it->second;
}
void set_lpc_override(int prec, long long n, int op, int colmode, int lpc) {
  std::lock_guard<std::mutex> lk(g_lpc_mu);
  if (lpc <= 0) g_lpc.erase(std::make_tuple(prec, n, op, colmode));
  else g_lpc[std::make_tuple(prec, n, op, colmode)] = lpc;
}
std::vector<std::array<long long, 5>> list_lpc_overrides() {
  std::lock_guard<std::mutex> lk(g_lpc_mu);
  std::vector<std::array<long long, 5>> v;
  for (auto &kv : g_lpc)
    v.push_back({std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first), std::get<3>(kv.first),
                 kv.second});
  return v;
}
std::vector<std::array<long long, 4>> list_pipe_overrides() {
  std::lock_guard<std::mutex> lk(g_lpc_mu);
  std::vector<std::array<long long, 4>> v;
  for (auto &kv : g_pipe)
    if (kv.second) v.push_back({std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first), kv.second});
  return v;
}
void clear_overrides() {
  for (auto &m : g_uneven_mode) m.store(-1);
  {
    std::lock_guard<std::mutex> lk(g_lpc_mu);
    g_lpc.clear();
    g_pipe.clear();
  }
  std::lock_guard<std::mutex> lk(g_sched_mu);
  g_sched.clear();
  g_sched_epoch.fetch_add(1);
}
int get_lpc_override(int prec, long long n, int op, int colmode) {
  std::lock_guard<std::mutex> lk(g_lpc_mu);
  auto it = g_lpc.find(std::make_tuple(prec, n, op, colmode));
  return it == g_lpc.end() ? 0 : it->second;
}

int choose_lpc(const DevProg &dp, const KArgs &a, int op, long long nlines, bool conv) {
  const int T = dp.lp.T;
  const size_t line_bytes = (size_t)spad_size(dp.n) * csize(dp.prec) + (conv ? 2 * csize(dp.prec) : 0);
  const size_t smax = max_smem_optin();
  const int colmode = (a.in.stride != 1 || a.out.stride != 1) ? 1 : 0;
  int lpc = get_lpc_override(dp.prec, dp.n, op, colmode);
  if (lpc <= 0) {
    // about 256 threads and at most half the shared memory per CTA, so two
    // CTAs share an SM: one's asynchronous prologue overlaps the other's
    // butterflies
    lpc = std::max(1, 256 / T);
    while (lpc > 1 && (size_t)lpc * line_bytes > smax / 2 - 1024) lpc--;
    if (colmode) {
      // columns: enough adjacent lines per CTA to fill 64-byte row segments
      const int want = dp.prec == F64 ? 4 : 8;
      const int cap = (int)std::min<size_t>(512 / T, smax / line_bytes);
      lpc = std::max(lpc, std::min(want, cap));
    }
    // small batches: fewer lines per CTA until the grid covers the SMs
    // (powers of two, the lines-per-CTA values the compiled kernels have)
    while (lpc > 1 && (nlines + lpc - 1) / lpc < num_sms() && (lpc & (lpc - 1)) == 0) lpc /= 2;
  }
  lpc = std::min(lpc, std::max(1, 512 / T));
  while (lpc > 1 && (size_t)lpc * line_bytes > smax) lpc--;
  if (lpc > nlines) lpc = (int)std::max<long long>(1, nlines);
  return lpc;
}

// True when every real pair (x[2j], x[2j+1]) of every line of a real Side is
// aligned to the pair size (so it moves as one vector copy).
bool pairs_aligned(const Side &s, int prec) {
  const long long pb = 2 * (long long)rsize(prec);
  return s.stride == 1 && !s.boff && ((uintptr_t)s.ptr % pb) == 0 && (s.dist_b % 2) == 0 &&
         (s.lpb.d == 1 || (s.dist_l % 2) == 0);
}

// Whether an op can read its first stage / write its last stage directly.
static bool op_fg(int op) {
  return op == OP_C2C || op == OP_C2C_TW || op == OP_R2C || op == OP_R2C_FULL || op == OP_RADER ||
         op == OP_BLUE || op == OP_SPECTRO;
}
static bool op_tg(int op) {
  return op == OP_C2C || op == OP_C2C_TW || op == OP_C2R || op == OP_R2C_FULL || op == OP_C2R_FULL ||
         op == OP_RADER || op == OP_BLUE;
}
// A side is column-like when adjacent lines sit closer than adjacent elements
// (a non-contiguous axis of a row-major array): threads then map across lines.
static bool side_col(const Side &s) {
  if (s.stride == 1) return false;
  const long long D = s.lpb.d > 1 ? s.dist_l : s.dist_b;
  return std::llabs(D) < std::llabs(s.stride);
}
int choose_flags(int op, const KArgs &a) {
  if (op == OP_FILTER_COL) return (side_col(a.in) ? GF_COLMAP : 0) | GF_FIRST_DIRECT | GF_LAST_DIRECT;
  // the packed real rows read (R2C) / write (C2R) pairs directly only when
  // they are unit-stride and pair-aligned
  if ((op == OP_R2C || op == OP_SPECTRO) && !(a.ic & GF_PAIR_ALIGNED)) return side_col(a.in) ? GF_COLMAP : 0;
  if (op == OP_C2R && !(a.ic & GF_PAIR_ALIGNED)) return side_col(a.out) ? GF_COLMAP : 0;
  if (op >= OP_RADER_FS1) return 0;  // gathers and scatters: row layout
  const bool fg = op_fg(op), tg = op_tg(op);
  const bool ic = side_col(a.in), oc = side_col(a.out);
  if (fg && tg) {
    if (ic == oc) return (ic ? GF_COLMAP : 0) | GF_FIRST_DIRECT | GF_LAST_DIRECT;
    return (ic ? GF_COLMAP : 0) | GF_FIRST_DIRECT;
  }
  if (fg) return (ic ? GF_COLMAP : 0) | GF_FIRST_DIRECT;
  if (tg) return (oc ? GF_COLMAP : 0) | GF_LAST_DIRECT;
  return 0;
}

// ---------------------------------------------------------------------------
// The TMA-fed persistent line kernel (k_pipe, pipe.cuh), for the plain
// complex, packed real forward and packed real inverse lines whenever an
// instance was built for the line's schedule and the layout suits it.  Off by
// default (gofft_set_tma_pipeline turns it on): on the 1024 x 1024 real round
// trip it measured no faster per launch than the one-tile-per-CTA kernels
// (its warps wait at the stage barriers instead of on the first stage's
// loads), and its one CTA per SM keeps the next L2 block's launch from
// overlapping the tail of the current one.
// ---------------------------------------------------------------------------
static std::atomic<int> g_pipe_on{0};
void set_tma_pipeline(int on) { g_pipe_on.store(on ? 1 : 0); }
int tma_pipeline() { return g_pipe_on.load(); }

// Programmatic dependent launch of the line kernels (k_line_ct, k_line):
// 0 off, 1 launched with programmatic stream serialization (each kernel
// waits for its predecessor in griddepcontrol.wait), 2 also triggering the
// next launch from every CTA's start.
static std::atomic<int> g_pdl{0};
void set_dependent_launch(int mode) { g_pdl.store(mode < 0 ? 0 : (mode > 2 ? 2 : mode)); }
int dependent_launch() { return g_pdl.load(); }

// The kernels' timeout word (set when a bounded wait gives up), one per
// device in the library image: its address comes from cudaGetSymbolAddress,
// so using it allocates nothing.
static __device__ int g_pipe_err;
static std::mutex g_pipe_err_mu;
static std::map<int, int *> g_pipe_err_addr;
static int *pipe_err_word() {
  const int d = cur_device();
  std::lock_guard<std::mutex> lk(g_pipe_err_mu);
  auto it = g_pipe_err_addr.find(d);
  if (it != g_pipe_err_addr.end()) return it->second;
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_pipe_err) != cudaSuccess) return nullptr;
  g_pipe_err_addr[d] = (int *)p;
  return (int *)p;
}
int pipe_status(bool clear) {
  int *w = pipe_err_word();
  if (!w) return set_err(3, "pipeline status word unavailable");
  int v = 0;
  GF_CK(cudaDeviceSynchronize());
  GF_CK(cudaMemcpy(&v, w, sizeof(int), cudaMemcpyDeviceToHost));
  if (v && clear) {
    const int zero = 0;
    GF_CK(cudaMemcpy(w, &zero, sizeof(int), cudaMemcpyHostToDevice));
  }
  return v ? set_err(4, "a pipelined line kernel's wait timed out") : 0;
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

static PipeInst pipe_instance(const DevProg &dp, int op, bool col) {
  const int *r = dp.lp.radix;
  switch (dp.prec) {
    case F64: return pipe_kernel_f64(op, dp.n, dp.lp.T, r, dp.lp.nst, col);
    case F32: return pipe_kernel_f32(op, dp.n, dp.lp.T, r, dp.lp.nst, col);
    default: return pipe_kernel_f32c(op, dp.n, dp.lp.T, r, dp.lp.nst, col);
  }
}

// Launches the line op on k_pipe when it applies: 1 (status in *rc) if it
// did, 0 when the caller should use the other line kernels.
static int try_pipe(int op, const DevProg &dp, KArgs a, long long nlines, cudaStream_t st, int *rc) {
  if (!g_pipe_on.load()) return 0;
  if (op != OP_C2C && op != OP_R2C && op != OP_C2R) return 0;
  const int n = dp.n;
  if (n < 16 || dp.lp.nst == 0) return 0;
  const size_t E = csize(dp.prec);
  bool col = false;
  if (op == OP_C2C) {
    col = side_col(a.in);
    if (col != side_col(a.out)) return 0;
    if (!col && (a.in.stride != 1 || a.out.stride != 1)) return 0;
  } else if (op == OP_R2C) {
    if (a.in.stride != 1 || !(a.ic & GF_PAIR_ALIGNED)) return 0;
  } else {
    if (a.in.stride != 1 || !(a.ic & GF_PAIR_ALIGNED) || (a.ic & GF_IC_MASK) != n + 1) return 0;
  }
  // the last stage indexes a line with 32-bit element offsets
  if (std::max(std::llabs(a.in.stride), std::llabs(a.out.stride)) * (long long)n >= (1ll << 31)) return 0;
  const PipeInst pi = pipe_instance(dp, op, col);
  if (!pi.fn || pi.smem > max_smem_optin()) return 0;
  PipeArgs pa{};
  pa.err = pipe_err_word();
  if (!pa.err) return 0;
  pa.spin_limit = 1u << 24;
  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  const int L = pi.lpc;
  if (col) {
    // lines are the columns of images: line b * ncols + c, adjacent columns
    // adjacent in memory
    const long long ncols = a.in.lpb.d;
    if (a.in.dist_l != 1 || a.in.boff || nlines % ncols != 0) return 0;
    const long long nimg = nlines / ncols;
    pa.ncols = (int)ncols;
    pa.tpb = (int)((ncols + L - 1) / L);
    pa.ntiles = nimg * pa.tpb;
    const int BR = n <= 256 ? n : 256;
    pa.box_rows = BR;
    pa.fill = PIPE_COL_ASYNC;
    // 2-D tensor copies when the images are the stacked rows of one array
    // whose row pitch and base meet the 16-byte rule
    const long long rows = nimg * n;
    auto enc = tensor_map_encoder();
    if (enc && a.in.dist_b == (long long)n * a.in.stride && n % BR == 0 && ((uintptr_t)a.in.ptr % 16) == 0 &&
        ((size_t)a.in.stride * E) % 16 == 0 && rows < (1ll << 31) && 2 * ncols < (1ll << 31)) {
      const cuuint64_t dims[2] = {(cuuint64_t)(2 * ncols), (cuuint64_t)rows};
      const cuuint64_t strides[1] = {(cuuint64_t)(a.in.stride * E)};
      const cuuint32_t box[2] = {(cuuint32_t)(2 * L), (cuuint32_t)BR};
      const cuuint32_t estr[2] = {1, 1};
      const CUresult r = enc(&map, dp.prec == F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                             2, a.in.ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r == CUDA_SUCCESS) pa.fill = PIPE_COL_TMA;
    }
  } else {
    pa.lp = op == OP_C2R ? n + 1 : n;
    pa.ntiles = (nlines + L - 1) / L;
    long long D = 0;
    pa.span = side_simple(a.in, D) ? D : 0;
    pa.fill = ((uintptr_t)a.in.ptr % 16) == 0 ? PIPE_ROW_BULK : PIPE_ROW_ASYNC;
  }
  // a persistent CTA pays off when it has tiles to overlap: with fewer than
  // two per SM the one-tile-per-CTA kernels fill the GPU better
  if (pa.ntiles < 2ll * num_sms()) return 0;
  a.lp = dp.lp;
  a.nlines = nlines;
  a.lpc = L;
  a.ndiv = FastDiv((uint32_t)n);
  a.lpcdiv = FastDiv((uint32_t)L);
  a.flags = (col ? GF_COLMAP : 0) | GF_LAST_DIRECT;
  if (int e = ensure_smem((KFn)pi.fn, pi.smem)) {
    *rc = e;
    return 1;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pi.fn, pi.threads, pi.smem);
  if (per_sm < 1) per_sm = 1;
  const long long grid = std::min<long long>(pa.ntiles, (long long)per_sm * num_sms());
  typedef void (*PipeFn)(KArgs, PipeArgs, CUtensorMap);
  count_launch();
  TimingRec rec;
  const bool timed = g_timing.load() != 0;
  if (timed) {
    cudaEventCreate(&rec.a);
    cudaEventCreate(&rec.b);
    cudaEventRecord(rec.a, st);
  }
  ((PipeFn)pi.fn)<<<(unsigned)grid, pi.threads, pi.smem, st>>>(a, pa, map);
  const cudaError_t e = cudaGetLastError();
  if (timed) {
    cudaEventRecord(rec.b, st);
    std::ostringstream k;
    k << op_name(op) << "/n=" << n << "/prec=" << dp.prec << "/pipe/lpc=" << L << "/T=" << dp.lp.T
      << "/fill=" << pa.fill;
    rec.key = k.str();
    rec.bytes = algo_bytes(op, dp, a, nlines);
    std::lock_guard<std::mutex> lk(g_tmu);
    g_trecs.push_back(rec);
  }
  *rc = e == cudaSuccess ? 0 : set_err(3, std::string("pipelined line kernel: ") + cudaGetErrorString(e));
  return 1;
}

// Two-CTA form: clusters of two CTAs, each holding half the convolution
// (persistent over the signals, one cluster per pair of SMs at most).
static int launch_rader_ip2(const DevProg &dp, KArgs a, long long nlines, cudaStream_t st) {
  int threads = 0;
  const void *f = dp.prec == F64 ? rader_ip2_kernel_f64(&threads)
                                 : (dp.prec == F32 ? rader_ip2_kernel_f32(&threads) : rader_ip2_kernel_f32c(&threads));
  a.lp = dp.lp;
  a.nlines = nlines;
  a.lpc = 1;
  a.ndiv = FastDiv((uint32_t)dp.n);
  a.lpcdiv = FastDiv(1);
  a.flags = 0;
  const size_t smem = (size_t)(dp.n / 2) * csize(dp.prec);
  if (int rc = ensure_smem((KFn)f, smem)) return rc;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3((unsigned)(2 * std::min<long long>(nlines, num_sms() / 2)));
  int clusters = 0;
  GF_CK(cudaOccupancyMaxActiveClusters(&clusters, f, &cfg));
  if (clusters < 1) return set_err(5, "two-CTA Rader kernel does not fit a pair of SMs");
  const long long full = std::min<long long>(nlines, clusters);
  const long long rounds = (nlines + full - 1) / full;
  cfg.gridDim = dim3((unsigned)(2 * ((nlines + rounds - 1) / rounds)));
  count_launch();
  TimingRec rec;
  const bool timed = g_timing.load() != 0;
  if (timed) {
    cudaEventCreate(&rec.a);
    cudaEventCreate(&rec.b);
    cudaEventRecord(rec.a, st);
  }
  void *args[] = {&a};
  GF_CK(cudaLaunchKernelExC(&cfg, f, args));
  if (timed) {
    cudaEventRecord(rec.b, st);
    std::ostringstream k;
    k << op_name(OP_RADER_IP) << "/p=" << a.ia << "/cl=" << dp.n << "/prec=" << dp.prec << "/T=" << threads
      << "/ctas=2";
    rec.key = k.str();
    rec.bytes = algo_bytes(OP_RADER_IP, dp, a, nlines);
    std::lock_guard<std::mutex> lk(g_tmu);
    g_trecs.push_back(rec);
  }
  return 0;
}

// The in-shared-memory Rader kernel: one CTA per signal (persistent over the
// signals), the convolution of length dp.n in dynamic shared memory.
static int launch_rader_ip(const DevProg &dp, KArgs a, long long nlines, cudaStream_t st) {
  if (dp.ctas == 2) return launch_rader_ip2(dp, a, nlines, st);
  int threads = 0;
  const void *f = dp.prec == F64 ? rader_ip_kernel_f64(&threads)
                                 : (dp.prec == F32 ? rader_ip_kernel_f32(&threads) : rader_ip_kernel_f32c(&threads));
  a.lp = dp.lp;
  a.nlines = nlines;
  a.lpc = 1;
  a.ndiv = FastDiv((uint32_t)dp.n);
  a.lpcdiv = FastDiv(1);
  a.flags = 0;
  const size_t smem = (size_t)dp.n * csize(dp.prec);
  if (int rc = ensure_smem((KFn)f, smem)) return rc;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, threads, smem);
  if (per_sm < 1) return set_err(5, "in-place Rader kernel does not fit an SM");
  // as many rounds of signals as the full grid needs, over as few CTAs as
  // give that many rounds (the rest of the SMs stay free for concurrent work)
  const long long full = std::min<long long>(nlines, (long long)per_sm * num_sms());
  const long long rounds = (nlines + full - 1) / full;
  const long long grid = (nlines + rounds - 1) / rounds;
  count_launch();
  TimingRec rec;
  const bool timed = g_timing.load() != 0;
  if (timed) {
    cudaEventCreate(&rec.a);
    cudaEventCreate(&rec.b);
    cudaEventRecord(rec.a, st);
  }
  ((KFn)f)<<<(unsigned)grid, threads, smem, st>>>(a);
  GF_CK(cudaGetLastError());
  if (timed) {
    cudaEventRecord(rec.b, st);
    std::ostringstream k;
    k << op_name(OP_RADER_IP) << "/p=" << a.ia << "/cl=" << dp.n << "/prec=" << dp.prec << "/T=" << threads
      << "/ctas=1";
    rec.key = k.str();
    rec.bytes = algo_bytes(OP_RADER_IP, dp, a, nlines);
    std::lock_guard<std::mutex> lk(g_tmu);
    g_trecs.push_back(rec);
  }
  return 0;
}

int launch_line(int op, const DevProg &dp, KArgs a, long long nlines, cudaStream_t st, int lpc,
                bool conv) {
  if (nlines <= 0) return 0;
  if (nlines >= (1ll << 31)) return set_err(5, "too many lines in one launch");
  if (op == OP_RADER_IP) return launch_rader_ip(dp, a, nlines, st);
  // tiled real intermediates are read and written by the one-tile-per-CTA
  // kernels only (the persistent variants do not know the layout)
  const bool tiled = (op == OP_R2C || op == OP_C2R) && (a.ic & GF_TILED);
  if (!conv && lpc <= 0 && !tiled) {
    int rc = 0;
    if (try_pipe(op, dp, a, nlines, st, &rc)) return rc;
  }
  a.lp = dp.lp;
  a.nlines = nlines;
  if (lpc <= 0) lpc = choose_lpc(dp, a, op, nlines, conv);
  a.lpc = lpc;
  a.ndiv = FastDiv((uint32_t)dp.n);
  a.lpcdiv = FastDiv((uint32_t)lpc);
  a.flags = choose_flags(op, a);
  // direct stages index a line with 32-bit element offsets
  if (std::max(std::llabs(a.in.stride), std::llabs(a.out.stride)) * (long long)dp.n >= (1ll << 31))
    a.flags &= GF_COLMAP;
  size_t smem = (size_t)lpc * spad_size(dp.n) * csize(dp.prec) + (conv ? 2 * lpc * csize(dp.prec) : 0);
  KFn f = nullptr;
  // the persistent double-buffered variant halves resident CTAs; measured
  // slower on the 1024/512-point lines, so it is opt-in (the autotuner's
  // pipe choice, gofft_set_pipelined)
  const bool no_pipe = tiled || !get_pipe_override(dp.prec, dp.n, op);
  long long grid = (nlines + lpc - 1) / lpc;
  bool pp = false;
  {
    // persistent double-buffered variant when two tile buffers fit
    if (!conv && !no_pipe && 2 * smem <= max_smem_optin() && grid > 2 * num_sms()) {
      f = kernel_ct_for(dp, op, lpc, true);
      if (f) {
        if (int rc = ensure_smem(f, 2 * smem)) return rc;
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)f, lpc * dp.lp.T, 2 * smem);
        if (per_sm < 1) per_sm = 1;
        grid = std::min<long long>(grid, (long long)per_sm * num_sms());
        smem *= 2;
        a.flags &= ~GF_FIRST_DIRECT;
        pp = true;
      }
    }
    if (!f) f = kernel_ct_for(dp, op, lpc, false);
  }
  if (!f) {
    // the run-time-schedule kernel has no direct stages
    f = kernel_for(dp.prec, dp.maxe, op);
    a.flags &= GF_COLMAP;
  }
  if (!f) return set_err(5, "no kernel instance for this precision/op");
  if (int rc = ensure_smem(f, smem)) return rc;
  count_launch();
  TimingRec rec;
  const bool timed = g_timing.load() != 0;
  if (timed) {
    cudaEventCreate(&rec.a);
    cudaEventCreate(&rec.b);
    cudaEventRecord(rec.a, st);
  }
  const int pdl = pp ? 0 : g_pdl.load();
  if (pdl) {
    if (pdl == 2) a.flags |= GF_PDL_TRIGGER;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)(lpc * dp.lp.T));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {&a};
    GF_CK(cudaLaunchKernelExC(&cfg, (const void *)f, args));
  } else {
    f<<<(unsigned)grid, lpc * dp.lp.T, smem, st>>>(a);
    GF_CK(cudaGetLastError());
  }
  if (timed) {
    cudaEventRecord(rec.b, st);
    std::ostringstream k;
    k << op_name(op) << "/n=" << dp.n << "/prec=" << dp.prec << "/lpc=" << lpc << "/T=" << dp.lp.T
      << "/flags=" << (a.flags & ~GF_PDL_TRIGGER);
    rec.key = k.str();
    rec.bytes = algo_bytes(op, dp, a, nlines);
    std::lock_guard<std::mutex> lk(g_tmu);
    g_trecs.push_back(rec);
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Exec1D
// ---------------------------------------------------------------------------
Exec1D::~Exec1D() {
  for (void *p : {(void *)tw4, (void *)perm, (void *)iperm, (void *)jj, spec, chirp, spec_ip})
    if (p) cudaFree(p);
}

size_t Exec1D::ws_bytes(long long nl) const {
  const size_t c = csize(prec);
  switch (kind) {
    case K_FOURSTEP: return 3 * (size_t)n * nl * c + 256;
    case K_RADER:
      if (fused || inplace) return 0;
      return (2 * (size_t)n + 2 * (size_t)cl + 2) * nl * c + 1024;
    case K_BLUE:
      if (fused) return 0;
      return 2 * (size_t)m * nl * c + 256 + sub->ws_bytes(nl);
    default: return 0;
  }
}

bool side_simple(const Side &s, long long &D) {
  if (s.boff) return false;
  if (s.lpb.d == 1) { D = s.dist_b; return true; }
  if (s.dist_b == (long long)s.lpb.d * s.dist_l) { D = s.dist_l; return true; }
  return false;
}

char *align256(char *p) { return (char *)(((uintptr_t)p + 255) & ~(uintptr_t)255); }


int Exec1D::exec(const Side &in, const Side &out, long long nl, int cji, int cjo, double scale,
                 void *ws, cudaStream_t st) const {
  if (nl <= 0 || n == 0) return 0;
  const size_t c = csize(prec);
  switch (kind) {
    case K_SINGLE: {
      KArgs a{};
      a.in = in;
      a.out = out;
      a.cj_in = cji;
      a.cj_out = cjo;
      a.scale = scale;
      return launch_line(OP_C2C, *prog, a, nl, st);
    }
    case K_FOURSTEP: {
      char *w = align256((char *)ws);
      Side src = in;
      long long Din = 0, Dout = 0;
      if (!side_simple(in, Din)) {
        EwArgs e{};
        e.nlines = nl;
        e.len = (int)n;
        e.ldst = (int)n;
        GF_CK(GF_PREC_CALL(prec, gather, w, in, e, st));
        src = contig(w, n);
        Din = n;
        w += (size_t)n * nl * c;
      }
      char *ws1 = w;
      w += (size_t)n * nl * c;
      // pass 1: n2 columns of length n1, twiddled by W_n^{n2 k1}
      KArgs a1{};
      a1.in = mk_side(src.ptr, Din, src.stride, n2 * src.stride, n2);
      a1.out = mk_side(ws1, n, 1, n2, n2);
      a1.cj_in = cji;
      a1.scale = 1.0;
      a1.aux0 = tw4;
      a1.ia = n;
      a1.ic = tw4_sh;
      if (int rc = launch_line(OP_C2C_TW, *p1, a1, nl * n2, st)) return rc;
      // pass 2: n1 rows of length n2, written transposed
      KArgs a2{};
      a2.in = mk_side(ws1, n, n2, 1, n1);
      a2.cj_out = cjo;
      a2.scale = scale;
      const bool direct = side_simple(out, Dout);
      char *ws2 = w;
      if (direct) a2.out = mk_side(out.ptr, Dout, out.stride, n1 * out.stride, n1);
      else a2.out = mk_side(ws2, n, 1, n1, n1);
      if (int rc = launch_line(OP_C2C, *p2, a2, nl * n1, st)) return rc;
      if (!direct) {
        EwArgs e{};
        e.nlines = nl;
        e.len = (int)n;
        e.scale = 1.0;
        GF_CK(GF_PREC_CALL(prec, scatter, out, ws2, e, st));
      }
      return 0;
    }
    case K_RADER: {
      if (fused) {
        KArgs a{};
        a.in = in;
        a.out = out;
        a.cj_in = cji;
        a.cj_out = cjo;
        a.scale = scale;
        a.aux0 = perm;
        a.aux1 = iperm;
        a.aux2 = spec;
        a.ia = n;
        a.ic = cyclic ? 0 : (int)(n - 1);
        return launch_line(OP_RADER, *prog, a, nl, st, 0, true);
      }
      if (inplace) {
        KArgs a{};
        a.in = in;
        a.out = out;
        a.cj_in = cji;
        a.cj_out = cjo;
        a.scale = scale;
        a.aux0 = perm;
        a.aux1 = iperm;
        a.aux2 = spec_ip;
        a.ia = n;
        a.ic = cyclic ? 0 : (int)(n - 1);
        return launch_line(OP_RADER_IP, *ipprog, a, nl, st);
      }
      return rader_two_pass(in, out, nl, cji, cjo, scale, ws, st);
    }
    case K_BLUE: {
      if (fused) {
        KArgs a{};
        a.in = in;
        a.out = out;
        a.cj_in = cji;
        a.cj_out = cjo;
        a.scale = scale;
        a.aux0 = chirp;
        a.aux2 = spec;
        a.ia = n;
        return launch_line(OP_BLUE, *prog, a, nl, st, 0, true);
      }
      char *w = align256((char *)ws);
      char *A = w;
      char *B = A + (size_t)m * nl * c;
      char *wsub = align256(B + (size_t)m * nl * c);
      EwArgs e{};
      e.nlines = nl;
      e.len = (int)n;
      e.ldst = (int)m;
      e.chirp = chirp;
      e.cj = cji;
      GF_CK(GF_PREC_CALL(prec, gather, A, in, e, st));
      if (int rc = sub->exec(contig(A, m), contig(B, m), nl, 0, 0, 1.0, wsub, st)) return rc;
      EwArgs e2{};
      e2.nlines = nl;
      e2.len = (int)m;
      GF_CK(GF_PREC_CALL(prec, spec_mul, B, spec, e2, st));
      if (int rc = sub->exec(contig(B, m), contig(A, m), nl, 0, 0, 1.0, wsub, st)) return rc;
      EwArgs e3{};
      e3.nlines = nl;
      e3.p = (int)n;
      e3.len = (int)m;
      e3.chirp = chirp;
      e3.cj = cjo;
      e3.scale = scale;
      GF_CK(GF_PREC_CALL(prec, blue_unchirp, out, A, e3, st));
      return 0;
    }
  }
  return set_err(1, "bad executor kind");
}

// Rader whose convolution runs as a two-pass split cl = n1 * n2 (the conv
// exec `sub` is K_FOURSTEP): four line-kernel passes (OpRaderFS1, OpRaderFS2,
// OpC2CTwiddle, OpRaderFS4) over two workspace buffers.
int Exec1D::rader_two_pass(const Side &in0, const Side &out0, long long nl, int cji, int cjo, double scale,
                           void *ws, cudaStream_t st) const {
  const size_t c = csize(prec);
  char *w = align256((char *)ws);
  Side in = in0, out = out0;
  long long Din = 0, Dout = 0;
  if (!(in.boff && in.lpb.d == 1) && !side_simple(in, Din)) {
    EwArgs e{};
    e.nlines = nl;
    e.len = (int)n;
    e.ldst = (int)n;
    GF_CK(GF_PREC_CALL(prec, gather, w, in, e, st));
    in = contig(w, n);
    Din = n;
    w += (size_t)n * nl * c;
  }
  char *outbuf = nullptr;
  if (!(out.boff && out.lpb.d == 1) && !side_simple(out, Dout)) {
    outbuf = w;
    w += (size_t)n * nl * c;
  }
  char *W1 = align256(w);
  char *W2 = W1 + (size_t)cl * nl * c;
  char *x0s = W2 + (size_t)cl * nl * c;
  char *dc = x0s + (size_t)nl * c;
  std::vector<RaderPhase> ph;
  rader_phases(in, Din, outbuf ? contig(outbuf, n) : out, outbuf ? n : Dout, nl, cji, cjo, scale, W1, W2, x0s,
               dc, ph);
  for (auto &q : ph)
    if (int rc = launch_line(q.op, *q.prog, q.a, q.nlines, st)) return rc;
  if (outbuf) {
    EwArgs e{};
    e.nlines = nl;
    e.len = (int)n;
    e.scale = 1.0;
    GF_CK(GF_PREC_CALL(prec, scatter, out, outbuf, e, st));
  }
  return 0;
}

// The four passes of rader_two_pass for signals addressed by `in` / `out`
// (signal s at s*D or boff[s], element stride), over workspaces W1, W2
// (cl per signal) and x0s, dc (one complex per signal).
void Exec1D::rader_phases(const Side &in, long long Din, const Side &out, long long Dout, long long nl, int cji,
                          int cjo, double scale, void *W1, void *W2, void *x0s, void *dc,
                          std::vector<RaderPhase> &ph) const {
  const Exec1D &cv = *sub;
  const long long N1 = cv.n1, N2 = cv.n2;
  const long long q = n - 1;
  auto sig_side = [&](const Side &s, long long D, long long lpb) {
    Side r = mk_side(s.ptr, D, 0, s.stride, lpb);
    r.boff = s.boff;
    return r;
  };
  RaderPhase f1{};
  f1.op = OP_RADER_FS1;
  f1.prog = cv.p1;
  f1.nlines = nl * N2;
  f1.a.in = sig_side(in, Din, N2);
  f1.a.out = mk_side(W1, cl, 1, N2, N2);
  f1.a.cj_in = cji;
  f1.a.scale = 1.0;
  f1.a.aux0 = perm;
  f1.a.aux1 = cv.tw4;
  f1.a.ic = cv.tw4_sh;
  f1.a.aux2 = x0s;
  f1.a.ia = cl;
  f1.a.ib = q;
  RaderPhase f2{};
  f2.op = OP_RADER_FS2;
  f2.prog = cv.p2;
  f2.nlines = nl * N1;
  f2.a.in = mk_side(W1, cl, N2, 1, N1);
  f2.a.out = mk_side(W2, cl, 1, N1, N1);
  f2.a.scale = 1.0;
  f2.a.aux0 = spec;
  f2.a.aux1 = x0s;
  f2.a.aux2 = dc;
  RaderPhase f3{};
  f3.op = OP_C2C_TW;
  f3.prog = cv.p1;
  f3.nlines = nl * N2;
  f3.a.in = mk_side(W2, cl, 1, N2, N2);
  f3.a.out = mk_side(W1, cl, 1, N2, N2);
  f3.a.scale = 1.0;
  f3.a.aux0 = cv.tw4;
  f3.a.ic = cv.tw4_sh;
  f3.a.ia = cl;
  RaderPhase f4{};
  f4.op = OP_RADER_FS4;
  f4.prog = cv.p2;
  f4.nlines = nl * N1;
  f4.a.in = mk_side(W1, cl, N2, 1, N1);
  f4.a.out = sig_side(out, Dout, N1);
  f4.a.cj_out = cjo;
  f4.a.scale = scale;
  f4.a.aux0 = iperm;
  f4.a.aux1 = x0s;
  f4.a.aux2 = dc;
  f4.a.ia = q;
  f4.a.ib = cyclic ? 0 : q;
  ph = {f1, f2, f3, f4};
}

std::string Exec1D::describe() const {
  std::ostringstream o;
  static const char *names[] = {"single", "fourstep", "rader", "bluestein"};
  o << "{\"n\":" << n << ",\"engine\":\"" << names[kind] << "\"";
  auto sched = [&](const DevProg &d) {
    std::ostringstream s;
    s << "{\"n\":" << d.n << ",\"T\":" << d.lp.T << ",\"maxe\":" << d.maxe << ",\"radices\":[";
    for (int i = 0; i < d.lp.nst; i++) s << (i ? "," : "") << d.lp.radix[i];
    s << "]}";
    return s.str();
  };
  if (kind == K_SINGLE && prog) o << ",\"prog\":" << sched(*prog);
  if (kind == K_FOURSTEP) o << ",\"n1\":" << n1 << ",\"n2\":" << n2 << ",\"p1\":" << sched(*p1) << ",\"p2\":" << sched(*p2);
  if (kind == K_RADER)
    o << ",\"g\":" << g << ",\"cl\":" << cl << ",\"cyclic\":" << cyclic << ",\"fused\":" << (fused ? 1 : 0)
      << ",\"inplace\":" << (inplace ? 1 : 0) << ",\"inplace_ctas\":" << (inplace ? ipprog->ctas : 0);
  if (kind == K_BLUE) o << ",\"m\":" << m << ",\"fused\":" << (fused ? 1 : 0);
  if ((kind == K_RADER || kind == K_BLUE) && fused && prog) o << ",\"prog\":" << sched(*prog);
  if ((kind == K_RADER || kind == K_BLUE) && !fused && sub) o << ",\"conv\":" << sub->describe();
  o << "}";
  return o.str();
}

// FP64 spectrum of a convolution kernel b (length L, device FP64), scaled by
// 1/L and stored in the precision's spectrum form.
static int make_spectrum(int prec, double2 *b, long long L, void **spec_out) {
  auto ex = get_exec(L, F64);
  if (!ex) return 3;
  double2 *B = nullptr;
  void *ws = nullptr;
  GF_CK(cudaMalloc(&B, L * sizeof(double2)));
  size_t wsb = ex->ws_bytes(1);
  if (wsb) GF_CK(cudaMalloc(&ws, wsb));
  int rc = ex->exec(contig(b, L), contig(B, L), 1, 0, 0, 1.0, ws, 0);
  if (rc == 0) {
    cudaError_t e = cudaMalloc(spec_out, L * spsize(prec));
    if (e == cudaSuccess) e = GF_PREC_CALL(prec, spectrum, *spec_out, B, 1.0 / (double)L, L, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) rc = set_err(3, std::string("spectrum: ") + cudaGetErrorString(e));
  }
  cudaFree(B);
  if (ws) cudaFree(ws);
  return rc;
}

// In-shared-memory Rader (rader_ip.cuh) for a convolution of length ex.cl
// that fits one CTA's shared memory: the stage list in decimation-in-
// frequency order (radix R_s, stride S_s = cl / (R_0 ... R_s)), the twiddle
// planes W_{R S}^{j m} (j < S, the Stockham table layout with ns = S), and
// the kernel spectrum permuted to the digit-reversed order the forward stages
// leave: A[k] at pos = sum_s m_s S_s for k = m_0 + R_0 m_1 + R_0 R_1 m_2 + ...
// A convolution too long for one CTA but even, whose first (power-of-two)
// radix is 2, 4 or 8 and whose half fits, runs on a cluster of two CTAs
// (k_rader_ip2), each holding half the line.
// Returns 0 when built, 1 when the length does not qualify, else an error.
static int build_rader_ip(Exec1D &ex) {
  const long long cl = ex.cl;
  const int prec = ex.prec;
  const std::vector<int> rad = gpu_radices(cl, 3);
  if (rad.empty() || (int)rad.size() > GF_MAXST) return 1;
  for (int R : rad)
    if (!rip_radix_ok(R)) return 1;
  // the kernels' static shared memory (two values) sits beside the line
  const size_t room = max_smem_optin() - 256;
  int ctas = 1;
  if ((size_t)cl * csize(prec) > room) {
    if (cl % 2 || !rip2_first_radix_ok(rad[0]) || (size_t)(cl / 2) * csize(prec) > room) return 1;
    ctas = 2;
  }
  auto dp = std::make_shared<DevProg>();
  dp->ctas = ctas;
  dp->n = (int)cl;
  dp->prec = prec;
  dp->device = cur_device();
  LineProg &lp = dp->lp;
  lp.n = (int)cl;
  lp.nst = (int)rad.size();
  lp.T = 1;
  lp.maxe = 16;
  StageTab tab{};
  tab.nst = lp.nst;
  long long S = cl, off = 0;
  for (int s = 0; s < lp.nst; s++) {
    S /= rad[s];
    lp.radix[s] = tab.radix[s] = rad[s];
    lp.ns[s] = tab.ns[s] = (int)S;
    lp.twoff[s] = tab.twoff[s] = (int)off;
    lp.nsdiv[s] = FastDiv((uint32_t)S);
    off += S * (rad[s] - 1);
  }
  GF_CK(cudaMalloc(&dp->tw, std::max<long long>(off, 1) * twsize(prec)));
  lp.tw = dp->tw;
  if (off > 0) GF_CK(GF_PREC_CALL(prec, stage_tw, dp->tw, tab, off, 0));
  // the spectrum in digit-reversed order (16-byte entries in every precision)
  std::vector<unsigned char> h((size_t)cl * 16), hp((size_t)cl * 16);
  GF_CK(cudaMemcpy(h.data(), ex.spec, h.size(), cudaMemcpyDeviceToHost));
  for (long long pos = 0; pos < cl; pos++) {
    long long rem = pos, k = 0, mult = 1;
    for (int s = 0; s < lp.nst; s++) {
      const long long m = rem / lp.ns[s];
      rem -= m * lp.ns[s];
      k += m * mult;
      mult *= lp.radix[s];
    }
    memcpy(&hp[(size_t)pos * 16], &h[(size_t)k * 16], 16);
  }
  GF_CK(cudaMalloc(&ex.spec_ip, hp.size()));
  GF_CK(cudaMemcpy(ex.spec_ip, hp.data(), hp.size(), cudaMemcpyHostToDevice));
  GF_CK(cudaStreamSynchronize(0));
  ex.ipprog = dp;
  ex.inplace = true;
  return 0;
}

static int build_exec(long long n, int prec, std::shared_ptr<Exec1D> &out) {
  auto ex = std::make_shared<Exec1D>();
  ex->n = n;
  ex->prec = prec;
  ex->device = cur_device();
  if (n < 0) return set_err(1, "negative length");
  if (n <= 1 || fits_single(n, prec)) {
    ex->kind = K_SINGLE;
    ex->prog = get_prog(n, prec);
    if (!ex->prog) return 3;
    out = ex;
    return 0;
  }
  if (smooth13(n)) {
    // four-step: n = n1 * n2 with both single-CTA lengths, n1 closest to sqrt
    long long best = 0;
    double bd = 1e300;
    for (long long d = 2; d * d <= n * 4 && d < n; d++) {
      if (n % d) continue;
      if (!fits_single(d, prec) || !fits_single(n / d, prec)) continue;
      const double dist = std::fabs(std::log((double)d) - 0.5 * std::log((double)n));
      if (dist < bd) { bd = dist; best = d; }
    }
    if (!best) return set_err(5, "length " + std::to_string(n) + " too long for a two-pass split");
    ex->kind = K_FOURSTEP;
    ex->n1 = best;
    ex->n2 = n / best;
    ex->p1 = get_prog(ex->n1, prec);
    ex->p2 = get_prog(ex->n2, prec);
    if (!ex->p1 || !ex->p2) return 3;
    // split twiddle table: S = 2^sh >= sqrt(n) entries W_n^e, then
    // ceil(n / S) entries W_n^(S j)
    int sh = 0;
    while ((1ll << (2 * sh)) < n) sh++;
    const long long S = 1ll << sh, J = (n + S - 1) / S;
    ex->tw4_sh = sh;
    GF_CK(cudaMalloc(&ex->tw4, (S + J) * twsize(prec)));
    GF_CK(GF_PREC_CALL(prec, roots, ex->tw4, n, S, 0));
    GF_CK(GF_PREC_CALL(prec, roots_step, (char *)ex->tw4 + S * twsize(prec), n, J, S, 0));
    GF_CK(cudaStreamSynchronize(0));
    out = ex;
    return 0;
  }
  if (n >= 700 && is_prime_ll(n)) {
    // Rader (rader.go:51-91)
    ex->kind = K_RADER;
    const long long q = n - 1;
    ex->g = primitive_root_ll(n);
    ex->cyclic = smooth13(q) ? 1 : 0;
    ex->cl = ex->cyclic ? q : best_conv_len(2 * q);
    GF_CK(cudaMalloc(&ex->perm, q * sizeof(int)));
    GF_CK(cudaMalloc(&ex->iperm, q * sizeof(int)));
    GF_CK(gen_rader_perm(ex->perm, ex->iperm, n, ex->g, 0));
    double2 *b = nullptr;
    GF_CK(cudaMalloc(&b, ex->cl * sizeof(double2)));
    GF_CK(gen_rader_kernel(b, ex->perm, n, ex->cl, ex->cyclic, 0));
    int rc = make_spectrum(prec, b, ex->cl, &ex->spec);
    cudaFree(b);
    if (rc) return rc;
    auto conv = get_exec(ex->cl, prec);
    if (!conv) return 3;
    if (conv->kind == K_SINGLE) {
      ex->fused = true;
      ex->prog = conv->prog;
    } else {
      ex->sub = conv;
      const int r = build_rader_ip(*ex);
      if (r > 1) return r;
    }
    out = ex;
    return 0;
  }
  // Bluestein (bluestein.go:28-48)
  ex->kind = K_BLUE;
  long long m = 1;
  while (m < 2 * n - 1) m <<= 1;
  ex->m = m;
  double2 *w = nullptr, *b = nullptr;
  GF_CK(cudaMalloc(&ex->jj, n * sizeof(long long)));
  GF_CK(cudaMalloc(&w, n * sizeof(double2)));
  GF_CK(cudaMalloc(&b, m * sizeof(double2)));
  GF_CK(gen_chirp(ex->jj, w, n, 0));
  GF_CK(gen_blue_kernel(b, w, n, m, 0));
  int rc = make_spectrum(prec, b, m, &ex->spec);
  if (rc == 0) {
    cudaError_t e = cudaMalloc(&ex->chirp, n * spsize(prec));
    if (e == cudaSuccess) e = GF_PREC_CALL(prec, spectrum, ex->chirp, w, 1.0, n, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) rc = set_err(3, std::string("chirp: ") + cudaGetErrorString(e));
  }
  cudaFree(w);
  cudaFree(b);
  if (rc) return rc;
  auto conv = get_exec(m, prec);
  if (!conv) return 3;
  if (conv->kind == K_SINGLE) {
    ex->fused = true;
    ex->prog = conv->prog;
  } else {
    ex->sub = conv;
  }
  out = ex;
  return 0;
}

std::shared_ptr<const Exec1D> get_exec(long long n, int prec) {
  static std::mutex mu;
  static std::map<std::tuple<int, long long, int, int>, std::shared_ptr<Exec1D>> cache;
  auto key = std::make_tuple(cur_device(), n, prec, sched_epoch());
  if (auto p = cache_get(cache, mu, key)) return p;
  // built outside the lock: prime lengths re-enter get_exec for their
  // convolution (the reference's cachedPlan does the same, plan.go:295-300)
  std::shared_ptr<Exec1D> p;
  if (build_exec(n, prec, p) != 0) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  cache[key] = p;
  return p;
}

// ---------------------------------------------------------------------------
// ExecReal
// ---------------------------------------------------------------------------
ExecReal::~ExecReal() {
  if (tw2) cudaFree(tw2);
  if (tw2_hi) cudaFree(tw2_hi);
}

size_t ExecReal::ws_bytes(long long nl) const {
  const size_t c = csize(prec);
  switch (mode) {
    case R_PACKED_MULTI: return (size_t)(n / 2) * nl * c + 256 + cx->ws_bytes(nl);
    case R_FULL_MULTI: return 2 * (size_t)n * nl * c + 256 + cx->ws_bytes(nl);
    default: return 0;
  }
}

int ExecReal::r2c(const Side &in, const Side &out, long long nl, void *ws, cudaStream_t st,
                  double wsc, long long tiled_rows) const {
  if (nl <= 0 || n == 0) return 0;
  const size_t c = csize(prec);
  const long long m = n / 2;
  if (tiled_rows > 0 && mode != R_PACKED_FUSED) return set_err(5, "tiled bins need a packed fused real plan");
  switch (mode) {
    case R_PACKED_FUSED: {
      KArgs a{};
      a.in = in;
      a.out = tiled_rows > 0 ? mk_side(out.ptr, 1, 0, 1, 1) : out;
      a.aux0 = tw2;
      a.aux1 = tw2_hi;
      a.scale = wsc != 0.0 ? wsc : 1.0;
      a.ic = (pairs_aligned(in, prec) ? GF_PAIR_ALIGNED : 0) | (wsc != 0.0 ? GF_EDGE_WEIGHT : 0) |
             (tiled_rows > 0 ? GF_TILED : 0);
      a.ib = tiled_rows;
      return launch_line(OP_R2C, *cx->prog, a, nl, st);
    }
    case R_FULL_FUSED: {
      KArgs a{};
      a.in = in;
      a.out = out;
      a.scale = wsc != 0.0 ? wsc : 1.0;
      a.ic = wsc != 0.0 ? GF_EDGE_WEIGHT : 0;
      return launch_line(OP_R2C_FULL, *cx->prog, a, nl, st);
    }
    case R_PACKED_MULTI: {
      if (in.stride != 1 || (in.dist_b % 2) || (in.dist_l % 2))
        return set_err(5, "packed real transform needs unit-stride rows with even distances");
      char *Z = align256((char *)ws);
      char *wsub = align256(Z + (size_t)m * nl * c);
      Side zin = mk_side(in.ptr, in.dist_b / 2, in.dist_l / 2, 1, in.lpb.d);
      if (int rc = cx->exec(zin, contig(Z, m), nl, 0, 0, 1.0, wsub, st)) return rc;
      GF_CK(GF_PREC_CALL(prec, untangle, out, Z, nl, (int)m, tw2, wsc, st));
      return 0;
    }
    case R_FULL_MULTI: {
      char *A = align256((char *)ws);
      char *B = A + (size_t)n * nl * c;
      char *wsub = align256(B + (size_t)n * nl * c);
      GF_CK(GF_PREC_CALL(prec, promote, A, in, nl, (int)n, st));
      if (int rc = cx->exec(contig(A, n), contig(B, n), nl, 0, 0, 1.0, wsub, st)) return rc;
      GF_CK(GF_PREC_CALL(prec, copy_bins, out, B, nl, (int)n, wsc, st));
      return 0;
    }
  }
  return set_err(1, "bad real mode");
}

int ExecReal::c2r(const Side &in, int nb, const Side &out, long long nl, double scale, void *ws,
                  cudaStream_t st, bool halve, long long tiled_rows) const {
  if (nl <= 0 || n == 0) return 0;
  const size_t c = csize(prec);
  const long long m = n / 2;
  if (tiled_rows > 0 && mode != R_PACKED_FUSED) return set_err(5, "tiled bins need a packed fused real plan");
  switch (mode) {
    case R_PACKED_FUSED: {
      KArgs a{};
      a.in = tiled_rows > 0 ? mk_side(in.ptr, 1, 0, 1, 1) : in;
      a.out = out;
      a.aux0 = tw2;
      a.aux1 = tw2_hi;
      a.ib = tiled_rows;
      a.ic = nb | (pairs_aligned(out, prec) ? GF_PAIR_ALIGNED : 0) | (halve ? GF_EDGE_WEIGHT : 0) |
             (tiled_rows > 0 ? GF_TILED : 0);
      a.scale = scale / (double)m;
      return launch_line(OP_C2R, *cx->prog, a, nl, st);
    }
    case R_FULL_FUSED: {
      KArgs a{};
      a.in = in;
      a.out = out;
      a.ic = nb | (halve ? GF_EDGE_WEIGHT : 0);
      a.scale = scale / (double)n;
      return launch_line(OP_C2R_FULL, *cx->prog, a, nl, st);
    }
    case R_PACKED_MULTI: {
      if (out.stride != 1 || (out.dist_b % 2) || (out.dist_l % 2))
        return set_err(5, "packed real transform needs unit-stride rows with even distances");
      char *Z = align256((char *)ws);
      char *wsub = align256(Z + (size_t)m * nl * c);
      GF_CK(GF_PREC_CALL(prec, reverse_untangle, Z, in, nl, (int)m, nb, tw2, halve ? 1 : 0, st));
      Side zout = mk_side(out.ptr, out.dist_b / 2, out.dist_l / 2, 1, out.lpb.d);
      return cx->exec(contig(Z, m), zout, nl, 0, 1, scale / (double)m, wsub, st);
    }
    case R_FULL_MULTI: {
      char *A = align256((char *)ws);
      char *B = A + (size_t)n * nl * c;
      char *wsub = align256(B + (size_t)n * nl * c);
      GF_CK(GF_PREC_CALL(prec, mirror, A, in, nl, (int)n, nb, halve ? 1 : 0, st));
      if (int rc = cx->exec(contig(A, n), contig(B, n), nl, 0, 0, 1.0, wsub, st)) return rc;
      GF_CK(GF_PREC_CALL(prec, take_real, out, B, nl, (int)n, scale / (double)n, st));
      return 0;
    }
  }
  return set_err(1, "bad real mode");
}

std::string ExecReal::describe() const {
  static const char *names[] = {"packed_fused", "packed_multi", "full_fused", "full_multi"};
  std::ostringstream o;
  o << "{\"n\":" << n << ",\"mode\":\"" << names[mode] << "\",\"complex\":" << cx->describe() << "}";
  return o.str();
}

static int build_real(long long n, int prec, std::shared_ptr<ExecReal> &out) {
  auto r = std::make_shared<ExecReal>();
  r->n = n;
  r->prec = prec;
  r->device = cur_device();
  if (n >= 2 && n % 2 == 0) {
    const long long m = n / 2;
    r->cx = get_exec(m, prec);
    if (!r->cx) return 3;
    r->mode = r->cx->kind == K_SINGLE ? R_PACKED_FUSED : R_PACKED_MULTI;
    GF_CK(cudaMalloc(&r->tw2, (m + 1) * twsize(prec)));
    GF_CK(GF_PREC_CALL(prec, roots, r->tw2, n, m + 1, 0));
    if (prec == F32C) {
      GF_CK(cudaMalloc(&r->tw2_hi, (m + 1) * twsize(F32)));
      GF_CK(GF_PREC_CALL(F32, roots, r->tw2_hi, n, m + 1, 0));
    }
    GF_CK(cudaStreamSynchronize(0));
  } else {
    r->cx = get_exec(n, prec);
    if (!r->cx) return 3;
    r->mode = r->cx->kind == K_SINGLE ? R_FULL_FUSED : R_FULL_MULTI;
  }
  out = r;
  return 0;
}

std::shared_ptr<const ExecReal> get_real(long long n, int prec) {
  static std::mutex mu;
  static std::map<std::tuple<int, long long, int, int>, std::shared_ptr<ExecReal>> cache;
  auto key = std::make_tuple(cur_device(), n, prec, sched_epoch());
  if (auto p = cache_get(cache, mu, key)) return p;
  std::shared_ptr<ExecReal> p;
  if (build_real(n, prec, p) != 0) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  cache[key] = p;
  return p;
}

}  // namespace gf
