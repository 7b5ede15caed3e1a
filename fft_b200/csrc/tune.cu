// tune.cu -- the autotuner and its wisdom.
//
// No counterpart in go-fft/fft (its plans are fixed by plan.go's router).
// For a plan shape the tuner times candidate settings on the device --
// the radix-schedule variant of every line length the plan uses, the lines
// per CTA of its line kernels, then the double-buffered persistent kernel
// per pass -- keeps the fastest, and leaves it set for plans created
// afterwards.  The settings are process-wide per
// (precision, length[, op, layout]), like FFTW's wisdom, and export to and
// import from a small JSON document.
#include <algorithm>
#include <cstring>
#include <functional>
#include <set>
#include <sstream>

#include "../../include/gofft.h"
#include "plan.cuh"

using namespace gf;

namespace {

// Deterministic fill (values in [-1, 1)) so the timed transforms see
// ordinary data.
__global__ void k_tune_fill(double *d, long long n, unsigned seed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + seed;
    z ^= z >> 31;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 29;
    d[i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}
__global__ void k_tune_fill32(float *d, long long n, unsigned seed) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + seed;
    z ^= z >> 31;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 29;
    d[i] = (float)((double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0);
  }
}

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

int fill(void *p, size_t bytes, int prec, cudaStream_t s) {
  if (prec == GOFFT_F64)
    k_tune_fill<<<592, 256, 0, s>>>((double *)p, (long long)(bytes / 8), 12345u);
  else
    k_tune_fill32<<<592, 256, 0, s>>>((float *)p, (long long)(bytes / 4), 12345u);
  return cudaGetLastError() == cudaSuccess ? 0 : set_err(GOFFT_ECUDA, "tuner fill failed");
}

// Median of `reps` timed runs after `warm` untimed ones (CUDA events on s).
int time_ms(const std::function<int(cudaStream_t)> &run, cudaStream_t s, int warm, int reps, double *ms) {
  for (int i = 0; i < warm; i++)
    if (int e = run(s)) return e;
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess) return set_err(GOFFT_ECUDA, "tuner event");
  if (cudaEventCreate(&b) != cudaSuccess) {
    cudaEventDestroy(a);
    return set_err(GOFFT_ECUDA, "tuner event");
  }
  std::vector<float> t;
  int rc = 0;
  for (int i = 0; i < reps && !rc; i++) {
    cudaEventRecord(a, s);
    rc = run(s);
    cudaEventRecord(b, s);
    if (!rc && cudaEventSynchronize(b) == cudaSuccess) {
      float v = 0;
      cudaEventElapsedTime(&v, a, b);
      t.push_back(v);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  if (t.empty()) return set_err(GOFFT_ECUDA, "tuner timing failed");
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return 0;
}

// One candidate evaluation: a fresh plan under the current settings, its
// forward and inverse transform on filled buffers.
int time_plan(int kind, int prec, const std::vector<long long> &shape, long long batch, cudaStream_t s,
              double *ms) {
  gofft_plan *p = nullptr;
  std::vector<int64_t> sh(shape.begin(), shape.end());
  if (int e = gofft_plan_create(kind, prec, sh.data(), (int)sh.size(), batch, 0, 0, 0, 0, &p)) return e;
  long long total = 1;
  for (long long v : shape) total *= v;
  const size_t rs = prec == GOFFT_F64 ? 8 : 4, cs = 2 * rs;
  const long long last = shape.back();
  const size_t cbytes =
      (size_t)batch * (kind == GOFFT_C2C ? total : total / last * (last / 2 + 1)) * cs;
  const size_t rbytes = kind == GOFFT_C2C ? cbytes : (size_t)batch * total * rs;
  DevBuf a, b;
  int rc = 0;
  if (cudaMalloc(&a.p, rbytes) != cudaSuccess || cudaMalloc(&b.p, cbytes) != cudaSuccess)
    rc = set_err(GOFFT_ENOMEM, "tuner buffers");
  if (!rc) rc = fill(a.p, rbytes, prec, s);
  if (!rc) {
    auto run = [&](cudaStream_t st) -> int {
      if (kind == GOFFT_C2C) {
        if (int e = gofft_exec_c2c(p, a.p, b.p, 0, st)) return e;
        return gofft_exec_c2c(p, b.p, a.p, 1, st);
      }
      if (int e = gofft_exec_r2c(p, a.p, b.p, st)) return e;
      return gofft_exec_c2r(p, b.p, 0, a.p, st);
    };
    rc = time_ms(run, s, 3, 9, ms);
  }
  cudaStreamSynchronize(s);
  gofft_plan_destroy(p);
  return rc;
}

// Line lengths a plan runs and the layout (column mode) of each pass.
struct Pass {
  long long n;  // program length
  int op;
  int colmode;
};

std::vector<Pass> plan_passes(int kind, const std::vector<long long> &shape) {
  std::vector<Pass> v;
  const int rank = (int)shape.size();
  if (kind == GOFFT_C2C) {
    for (int a = 0; a < rank; a++)
      if (shape[a] > 1) v.push_back({shape[a], OP_C2C, a < rank - 1 ? 1 : 0});
    return v;
  }
  const long long last = shape.back();
  const bool packed = last >= 2 && last % 2 == 0;
  const long long nl = packed ? last / 2 : last;
  v.push_back({nl, packed ? OP_R2C : OP_R2C_FULL, 0});
  v.push_back({nl, packed ? OP_C2R : OP_C2R_FULL, 0});
  if (rank == 2 && shape[0] > 1) v.push_back({shape[0], OP_C2C, 1});
  return v;
}

std::string wisdom_json() {
  std::ostringstream o;
  o << "{\"gofft_wisdom\":1,\"schedule\":[";
  bool f = true;
  for (auto &e : list_sched_variants()) {
    o << (f ? "" : ",") << "[" << e[0] << "," << e[1] << "," << e[2] << "]";
    f = false;
  }
  o << "],\"lpc\":[";
  f = true;
  for (auto &e : list_lpc_overrides()) {
    o << (f ? "" : ",") << "[" << e[0] << "," << e[1] << "," << e[2] << "," << e[3] << "," << e[4] << "]";
    f = false;
  }
  o << "],\"pipe\":[";
  f = true;
  for (auto &e : list_pipe_overrides()) {
    o << (f ? "" : ",") << "[" << e[0] << "," << e[1] << "," << e[2] << "," << e[3] << "]";
    f = false;
  }
  o << "],\"uneven\":[";
  f = true;
  for (int pr = 0; pr < 3; pr++) {
    const int m = get_uneven_mode(pr);
    if (m < 0) continue;
    o << (f ? "" : ",") << "[" << pr << "," << m << "]";
    f = false;
  }
  o << "]}";
  return o.str();
}

int64_t put_string(const std::string &s, char *buf, int64_t cap) {
  if (buf && cap > 0) {
    const size_t k = std::min<size_t>(s.size(), (size_t)cap - 1);
    memcpy(buf, s.data(), k);
    buf[k] = 0;
  }
  return (int64_t)s.size();
}

// Parses the array of integer tuples after "key": [[a,b,...],...].  Returns
// false on a malformed document.
bool parse_tuples(const std::string &js, const char *key, size_t width, std::vector<std::vector<long long>> &out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t i = js.find(k);
  if (i == std::string::npos) return true;  // absent: nothing to import
  i = js.find('[', i + k.size());
  if (i == std::string::npos) return false;
  i++;
  for (;;) {
    while (i < js.size() && (js[i] == ' ' || js[i] == ',' || js[i] == '\n')) i++;
    if (i >= js.size()) return false;
    if (js[i] == ']') return true;
    if (js[i] != '[') return false;
    i++;
    std::vector<long long> t;
    for (;;) {
      while (i < js.size() && (js[i] == ' ' || js[i] == ',')) i++;
      if (i >= js.size()) return false;
      if (js[i] == ']') {
        i++;
        break;
      }
      char *end = nullptr;
      const long long v = strtoll(js.c_str() + i, &end, 10);
      if (end == js.c_str() + i) return false;
      t.push_back(v);
      i = (size_t)(end - js.c_str());
    }
    if (t.size() != width) return false;
    out.push_back(t);
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" int64_t gofft_autotune(int kind, int precision, const int64_t *shape, int rank, int64_t batch,
                                  char *wisdom, int64_t cap) {
  if (!shape || rank < 1 || batch < 1 || (kind != GOFFT_C2C && kind != GOFFT_R2C) || precision < 0 ||
      precision > 2) {
    set_err(GOFFT_EINVAL, "bad autotune arguments");
    return -GOFFT_EINVAL;
  }
  std::vector<long long> sh(shape, shape + rank);
  for (long long v : sh)
    if (v <= 0) {
      set_err(GOFFT_EINVAL, "fft: shape lengths must be positive");
      return -GOFFT_EINVAL;
    }
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    set_err(GOFFT_ECUDA, "tuner stream");
    return -GOFFT_ECUDA;
  }
  const std::vector<Pass> passes = plan_passes(kind, sh);
  std::vector<long long> lens;
  for (auto &ps : passes)
    if (std::find(lens.begin(), lens.end(), ps.n) == lens.end() && fits_single(ps.n, precision))
      lens.push_back(ps.n);
  int rc = 0;
  double best = 0;
  rc = time_plan(kind, precision, sh, batch, s, &best);
  // 1. schedule variants: coordinate descent over the distinct lengths
  const int nvar = precision == GOFFT_F64 ? 2 : 3;
  for (size_t li = 0; li < lens.size() && !rc; li++) {
    const long long n = lens[li];
    int keep = get_sched_variant(precision, n);
    for (int v = 0; v < nvar; v++) {
      if (v == keep) continue;
      const int prev = keep;
      set_sched_variant(precision, n, v);
      double t = 0;
      if (time_plan(kind, precision, sh, batch, s, &t) == 0 && t < best * 0.98) {
        best = t;
        keep = v;
      } else {
        set_sched_variant(precision, n, prev);
      }
    }
  }
  // 2. lines per CTA of each pass (the kernels pick it at launch)
  for (size_t pi = 0; pi < passes.size() && !rc; pi++) {
    const Pass &ps = passes[pi];
    auto prog = get_prog(ps.n, precision);
    if (!prog) continue;
    const int T = prog->lp.T;
    const int cur = get_lpc_override(precision, ps.n, ps.op, ps.colmode);
    int keep = cur;
    for (int l : {1, 2, 4, 8, 16, 32}) {
      if (l * T > 512 || l == cur) continue;
      set_lpc_override(precision, ps.n, ps.op, ps.colmode, l);
      double t = 0;
      if (time_plan(kind, precision, sh, batch, s, &t) == 0 && t < best * 0.98) {
        best = t;
        keep = l;
      }
    }
    set_lpc_override(precision, ps.n, ps.op, ps.colmode, keep);
  }
  // 3. the persistent double-buffered kernel per pass (prefetches the next
  //    tile while the current one is transformed)
  for (size_t pi = 0; pi < passes.size() && !rc; pi++) {
    const Pass &ps = passes[pi];
    if (get_pipe_override(precision, ps.n, ps.op)) continue;
    set_pipe_override(precision, ps.n, ps.op, 1);
    double t = 0;
    if (time_plan(kind, precision, sh, batch, s, &t) == 0 && t < best * 0.98) best = t;
    else set_pipe_override(precision, ps.n, ps.op, 0);
  }
  cudaStreamDestroy(s);
  if (rc) return -rc;
  return put_string(wisdom_json(), wisdom, cap);
}

extern "C" int64_t gofft_autotune_uneven(int precision, const int64_t *lengths, int64_t count, char *wisdom,
                                         int64_t cap) {
  if (!lengths || count < 1 || precision < 0 || precision > 2) {
    set_err(GOFFT_EINVAL, "bad autotune arguments");
    return -GOFFT_EINVAL;
  }
  long long total = 0;
  std::set<long long> cls;
  for (int64_t i = 0; i < count; i++) {
    if (lengths[i] < 0) {
      set_err(GOFFT_EINVAL, "negative length");
      return -GOFFT_EINVAL;
    }
    total += lengths[i];
    if (lengths[i] > 1 && fits_single(lengths[i], precision)) cls.insert(lengths[i]);
  }
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    set_err(GOFFT_ECUDA, "tuner stream");
    return -GOFFT_ECUDA;
  }
  const size_t bytes = (size_t)std::max<long long>(1, total) * (precision == GOFFT_F64 ? 16 : 8);
  DevBuf a, b;
  int rc = 0;
  if (cudaMalloc(&a.p, bytes) != cudaSuccess || cudaMalloc(&b.p, bytes) != cudaSuccess)
    rc = set_err(GOFFT_ENOMEM, "tuner buffers");
  if (!rc) rc = fill(a.p, bytes, precision, s);
  auto measure = [&](double *ms) -> int {
    gofft_uneven *u = nullptr;
    if (int e = gofft_uneven_create(precision, lengths, count, nullptr, nullptr, &u)) return e;
    auto run = [&](cudaStream_t st) -> int { return gofft_uneven_exec(u, a.p, b.p, 0, st); };
    int e = time_ms(run, s, 3, 9, ms);
    cudaStreamSynchronize(s);
    if (!e && gofft_uneven_status(u) != GOFFT_OK) e = set_err(GOFFT_ETIMEOUT, "tuner run timed out");
    gofft_uneven_destroy(u);
    return e;
  };
  double best = 0;
  if (!rc) rc = measure(&best);
  const int nvar = 2;  // uneven batches build variants 0 and 1 only
  for (long long n : cls) {
    if (rc) break;
    int keep = get_sched_variant(precision, n);
    for (int v = 0; v < nvar; v++) {
      if (v == keep) continue;
      const int prev = keep;
      set_sched_variant(precision, n, v);
      double t = 0;
      if (measure(&t) == 0 && t < best * 0.98) {
        best = t;
        keep = v;
      } else {
        set_sched_variant(precision, n, prev);
      }
    }
  }
  // persistent launch or one launch per phase
  if (!rc) {
    const int cur = get_uneven_mode(precision);
    set_uneven_mode(precision, cur == 0 ? 1 : 0);
    double t = 0;
    if (measure(&t) == 0 && t < best * 0.98) best = t;
    else set_uneven_mode(precision, cur);
  }
  cudaStreamDestroy(s);
  if (rc) return -rc;
  return put_string(wisdom_json(), wisdom, cap);
}

extern "C" int64_t gofft_wisdom_export(char *buf, int64_t cap) { return put_string(wisdom_json(), buf, cap); }

extern "C" int gofft_wisdom_import(const char *json) {
  if (!json) return set_err(GOFFT_EINVAL, "null wisdom");
  const std::string js(json);
  if (js.find("\"gofft_wisdom\"") == std::string::npos) return set_err(GOFFT_EINVAL, "not gofft wisdom");
  std::vector<std::vector<long long>> sc, lp, pp, un;
  if (!parse_tuples(js, "schedule", 3, sc) || !parse_tuples(js, "lpc", 5, lp) || !parse_tuples(js, "pipe", 4, pp) ||
      !parse_tuples(js, "uneven", 2, un))
    return set_err(GOFFT_EINVAL, "malformed wisdom");
  for (auto &t : un)
    if (t[0] < 0 || t[0] > 2 || t[1] < 0 || t[1] > 1) return set_err(GOFFT_EINVAL, "bad uneven entry");
  for (auto &t : sc)
    if (t[0] < 0 || t[0] > 2 || t[1] < 1 || t[2] < 0 || t[2] > 2) return set_err(GOFFT_EINVAL, "bad schedule entry");
  for (auto &t : lp)
    if (t[0] < 0 || t[0] > 2 || t[1] < 1 || t[2] < 0 || t[2] >= OP_COUNT || t[4] < 0 || t[4] > 512)
      return set_err(GOFFT_EINVAL, "bad lpc entry");
  for (auto &t : pp)
    if (t[0] < 0 || t[0] > 2 || t[1] < 1 || t[2] < 0 || t[2] >= OP_COUNT) return set_err(GOFFT_EINVAL, "bad pipe entry");
  for (auto &t : sc) set_sched_variant((int)t[0], t[1], (int)t[2]);
  for (auto &t : lp) set_lpc_override((int)t[0], t[1], (int)t[2], (int)t[3], (int)t[4]);
  for (auto &t : pp) set_pipe_override((int)t[0], t[1], (int)t[2], (int)t[3]);
  for (auto &t : un) set_uneven_mode((int)t[0], (int)t[1]);
  return GOFFT_OK;
}

extern "C" int gofft_wisdom_forget(void) {
  clear_overrides();
  return GOFFT_OK;
}
