// uneven.cu -- many 1-D complex transforms of different lengths in one
// persistent launch.
//
// The signals are grouped by length.  Each length's executor is lowered to a
// list of phases (one line op over a number of tiles): one phase for a length
// that fits one CTA (and for a Rader or Bluestein transform whose convolution
// fits one CTA, and for a Rader transform whose convolution fits one CTA's
// shared memory), two for the four-step split, four for Rader over a two-pass
// convolution.  Phases are ordered by dependency level (every first phase,
// then every second phase, ...) and executed by k_persist, whose CTAs claim
// (phase, tile) items from a counter; a phase waits, with a bounded spin, for
// the phase it depends on.  The same phases can also be launched one kernel
// each (the per-phase mode: compiled-schedule kernels where they exist, the
// length classes spread over four streams so independent classes overlap);
// the autotuner picks the faster mode.
#include <algorithm>
#include <cstring>
#include <map>
#include <sstream>

#include "../../include/gofft.h"
#include "kernels.cuh"
#include "plan.cuh"

using namespace gf;

#define GF_CK(x)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess)                                                              \
      return set_err(GOFFT_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_));     \
  } while (0)

namespace {
// Placeholders for the caller's packed input / output, patched per call.
char g_in_tag, g_out_tag;
}  // namespace

struct gofft_uneven {
  int prec = 0, device = 0, persistent = 1;
  long long count = 0;
  struct Cls {
    long long n = 0;
    std::vector<long long> sig;
    std::shared_ptr<const Exec1D> ex;
    long long *d_ioff = nullptr, *d_ooff = nullptr;
  };
  std::vector<Cls> cls;
  std::vector<PhaseDesc> ph[2];        // forward, inverse (user pointers as tags)
  std::vector<int> ph_level;
  std::vector<int> ph_lane;            // per-phase launches: stream index (by class)
  std::vector<int> launch_order;       // per-phase launches: phases in class order
  std::vector<std::shared_ptr<DevProg>> ph_prog;
  static constexpr int kLanes = 4;     // per-phase launches: classes spread over these streams
  cudaStream_t lane[kLanes] = {};      // lane[0] unused (the caller's stream)
  cudaEvent_t ev_fork = nullptr, ev_join[kLanes] = {};
  PhaseDesc *d_ph[2] = {nullptr, nullptr};
  PhaseDesc *h_pinned = nullptr;       // staging for pointer patches
  void *ws = nullptr;
  size_t ws_bytes = 0;
  unsigned long long *d_ctr = nullptr;  // counter, then done[nph], err
  int nph = 0, block = 0;
  long long total = 0;
  size_t smem = 0;
  int grid = 0;
  long long spin_limit = 1ll << 24;
  int extra_wait = 0;                  // test hook: dependencies that never complete
  const void *last_in[2] = {nullptr, nullptr};
  void *last_out[2] = {nullptr, nullptr};
  ~gofft_uneven() {
    for (auto &c : cls) {
      if (c.d_ioff) cudaFree(c.d_ioff);
      if (c.d_ooff) cudaFree(c.d_ooff);
    }
    for (auto p : d_ph)
      if (p) cudaFree(p);
    if (h_pinned) cudaFreeHost(h_pinned);
    if (ws) cudaFree(ws);
    if (d_ctr) cudaFree(d_ctr);
    for (int k = 1; k < kLanes; k++) {
      if (lane[k]) cudaStreamDestroy(lane[k]);
      if (ev_join[k]) cudaEventDestroy(ev_join[k]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
  }
};

// The persistent kernel of a precision (instantiated with the compiled
// schedules it dispatches to, in the precision's own translation unit).
using PersistFn = void (*)(const PhaseDesc *, int, long long, unsigned long long *, int *, int *, long long);
static const void *persist_fn(int prec) {
  return prec == F64 ? persist_kernel_f64() : prec == F32 ? persist_kernel_f32() : persist_kernel_f32c();
}

static int *done_ptr(gofft_uneven *u) { return reinterpret_cast<int *>(u->d_ctr + 1); }
static int *err_ptr(gofft_uneven *u) { return done_ptr(u) + u->nph; }

static Side tag_side(char *tag, const long long *boff, long long dist_l, long long stride, long long lpb) {
  Side s = mk_side(tag, 0, dist_l, stride, lpb);
  s.boff = boff;
  return s;
}

// Appends the phases of one length class.  Sides on the caller's buffers
// carry the tags; workspace regions are carved from *wsoff.
static int add_class(gofft_uneven *u, gofft_uneven::Cls &c, size_t *wsoff, std::vector<PhaseDesc> &out,
                     std::vector<int> &level, std::vector<std::shared_ptr<DevProg>> &progs) {
  const Exec1D &e = *c.ex;
  const long long cnt = (long long)c.sig.size();
  const size_t cs = csize(u->prec);
  auto carve = [&](size_t bytes) {
    const size_t off = (*wsoff + 255) & ~(size_t)255;
    *wsoff = off + bytes;
    return (char *)nullptr + off;  // offset; rebased once the workspace exists
  };
  auto push = [&](int op, const std::shared_ptr<DevProg> &prog, KArgs a, long long nlines, int dep, int lvl,
                  bool conv) {
    PhaseDesc p{};
    a.lp = prog->lp;
    a.nlines = nlines;
    // the in-shared-memory Rader works on one signal per item
    a.lpc = op == OP_RADER_IP ? 1 : choose_lpc(*prog, a, op, nlines, conv);
    a.ndiv = FastDiv((uint32_t)prog->n);
    a.lpcdiv = FastDiv((uint32_t)a.lpc);
    a.flags = choose_flags(op, a) & GF_COLMAP;
    p.a = a;
    p.op = op;
    p.dep = dep;
    p.ntiles = (nlines + a.lpc - 1) / a.lpc;
    out.push_back(p);
    level.push_back(lvl);
    progs.push_back(prog);
    return (int)out.size() - 1;
  };
  const Side in1 = tag_side(&g_in_tag, c.d_ioff, 0, 1, 1);
  const Side out1 = tag_side(&g_out_tag, c.d_ooff, 0, 1, 1);
  if (e.kind == K_SINGLE) {
    KArgs a{};
    a.in = in1;
    a.out = out1;
    a.scale = 1.0;
    push(OP_C2C, e.prog, a, cnt, -1, 0, false);
    return 0;
  }
  if (e.kind == K_FOURSTEP) {
    // L2 blocks of signals (at most 48 MB of intermediate each), two phases
    // per block: launched one launch per phase, a block's second pass reads
    // its intermediate from L2
    const long long kb = std::max<long long>(1, std::min<long long>(cnt, (48ll << 20) / (e.n * (long long)cs)));
    for (long long b0 = 0; b0 < cnt; b0 += kb) {
      const long long nb = std::min(kb, cnt - b0);
      char *w = carve((size_t)e.n * nb * cs);
      KArgs a1{};
      a1.in = tag_side(&g_in_tag, c.d_ioff + b0, 1, e.n2, e.n2);
      a1.out = mk_side(w, e.n, 1, e.n2, e.n2);
      a1.scale = 1.0;
      a1.aux0 = e.tw4;
      a1.ia = e.n;
      a1.ic = e.tw4_sh;
      const int p1 = push(OP_C2C_TW, e.p1, a1, nb * e.n2, -1, 0, false);
      KArgs a2{};
      a2.in = mk_side(w, e.n, e.n2, 1, e.n1);
      a2.out = tag_side(&g_out_tag, c.d_ooff + b0, 1, e.n1, e.n1);
      a2.scale = 1.0;
      push(OP_C2C, e.p2, a2, nb * e.n1, p1, 1, false);
    }
    return 0;
  }
  if (e.kind == K_RADER && e.fused) {
    KArgs a{};
    a.in = in1;
    a.out = out1;
    a.scale = 1.0;
    a.aux0 = e.perm;
    a.aux1 = e.iperm;
    a.aux2 = e.spec;
    a.ia = e.n;
    a.ic = e.cyclic ? 0 : (int)(e.n - 1);
    push(OP_RADER, e.prog, a, cnt, -1, 0, true);
    return 0;
  }
  if (e.kind == K_BLUE && e.fused) {
    KArgs a{};
    a.in = in1;
    a.out = out1;
    a.scale = 1.0;
    a.aux0 = e.chirp;
    a.aux2 = e.spec;
    a.ia = e.n;
    push(OP_BLUE, e.prog, a, cnt, -1, 0, true);
    return 0;
  }
  // (the two-CTA form is not a persistent-kernel phase: those classes take
  // the four passes below)
  if (e.kind == K_RADER && e.inplace && e.ipprog->ctas == 1) {
    KArgs a{};
    a.in = in1;
    a.out = out1;
    a.scale = 1.0;
    a.aux0 = e.perm;
    a.aux1 = e.iperm;
    a.aux2 = e.spec_ip;
    a.ia = e.n;
    a.ic = e.cyclic ? 0 : (int)(e.n - 1);
    push(OP_RADER_IP, e.ipprog, a, cnt, -1, 0, false);
    return 0;
  }
  if (e.kind == K_RADER && e.sub && e.sub->kind == K_FOURSTEP) {
    char *W1 = carve((size_t)e.cl * cnt * cs);
    char *W2 = carve((size_t)e.cl * cnt * cs);
    char *x0s = carve((size_t)cnt * cs);
    char *dc = carve((size_t)cnt * cs);
    std::vector<RaderPhase> rp;
    e.rader_phases(in1, 0, out1, 0, cnt, 0, 0, 1.0, W1, W2, x0s, dc, rp);
    int prev = -1;
    for (size_t i = 0; i < rp.size(); i++) prev = push(rp[i].op, rp[i].prog, rp[i].a, rp[i].nlines, prev, (int)i, false);
    return 0;
  }
  return set_err(GOFFT_EUNSUPPORTED, "length " + std::to_string(c.n) + " has no persistent schedule");
}

// Replaces the tags and workspace offsets of one side.
static void rebase_side(Side &s, char *ws, const void *in, void *out) {
  if (s.ptr == &g_in_tag) s.ptr = (void *)in;
  else if (s.ptr == &g_out_tag) s.ptr = out;
  else if ((uintptr_t)s.ptr < ((uintptr_t)1 << 40) && ws) s.ptr = ws + (uintptr_t)s.ptr;
}
static void rebase_aux(const void *&p, char *ws, size_t wsb) {
  if ((uintptr_t)p < wsb + 256 && p != nullptr) p = ws + (uintptr_t)p;
}

extern "C" int gofft_uneven_create(int precision, const int64_t *lengths, int64_t count, const int64_t *in_offsets,
                                   const int64_t *out_offsets, gofft_uneven **out) {
  SchedCap cap(1);  // every class runs in the persistent kernel's 16-element registers
  if (!out || !lengths || count <= 0) return set_err(GOFFT_EINVAL, "bad uneven batch arguments");
  *out = nullptr;
  if (precision < 0 || precision > 2) return set_err(GOFFT_EINVAL, "bad precision");
  std::unique_ptr<gofft_uneven> u(new gofft_uneven());
  u->prec = precision;
  if (get_uneven_mode(precision) == 0) u->persistent = 0;  // the tuner's choice
  u->count = count;
  cudaGetDevice(&u->device);
  std::vector<long long> ioff(count), ooff(count);
  long long acc = 0;
  for (int64_t i = 0; i < count; i++) {
    if (lengths[i] < 1) return set_err(GOFFT_EINVAL, "uneven batch lengths must be positive");
    ioff[i] = in_offsets ? in_offsets[i] : acc;
    ooff[i] = out_offsets ? out_offsets[i] : ioff[i];
    acc += lengths[i];
  }
  std::map<long long, size_t> byn;
  for (int64_t i = 0; i < count; i++) {
    auto it = byn.find(lengths[i]);
    if (it == byn.end()) {
      byn[lengths[i]] = u->cls.size();
      u->cls.emplace_back();
      u->cls.back().n = lengths[i];
      it = byn.find(lengths[i]);
    }
    u->cls[it->second].sig.push_back(i);
  }
  // per-class offset tables and executors
  for (auto &c : u->cls) {
    c.ex = get_exec(c.n, precision);
    if (!c.ex) return GOFFT_ECUDA;
    std::vector<long long> a, b;
    for (long long s : c.sig) {
      a.push_back(ioff[s]);
      b.push_back(ooff[s]);
    }
    GF_CK(cudaMalloc(&c.d_ioff, a.size() * sizeof(long long)));
    GF_CK(cudaMalloc(&c.d_ooff, b.size() * sizeof(long long)));
    GF_CK(cudaMemcpy(c.d_ioff, a.data(), a.size() * sizeof(long long), cudaMemcpyHostToDevice));
    GF_CK(cudaMemcpy(c.d_ooff, b.data(), b.size() * sizeof(long long), cudaMemcpyHostToDevice));
  }
  // phases (forward), in per-class order first
  std::vector<PhaseDesc> raw;
  std::vector<int> lvl;
  std::vector<std::shared_ptr<DevProg>> progs;
  size_t wsoff = 0;
  // classes spread over the per-phase lanes, largest first (round robin)
  std::vector<size_t> by_size(u->cls.size());
  for (size_t i = 0; i < by_size.size(); i++) by_size[i] = i;
  std::stable_sort(by_size.begin(), by_size.end(), [&](size_t x, size_t y) {
    return u->cls[x].n * (long long)u->cls[x].sig.size() > u->cls[y].n * (long long)u->cls[y].sig.size();
  });
  std::vector<int> cls_lane(u->cls.size()), raw_lane;
  std::vector<long long> raw_len;  // class length of each phase
  for (size_t r = 0; r < by_size.size(); r++) cls_lane[by_size[r]] = (int)(r % gofft_uneven::kLanes);
  for (size_t ci = 0; ci < u->cls.size(); ci++) {
    const size_t first = raw.size();
    if (int rc = add_class(u.get(), u->cls[ci], &wsoff, raw, lvl, progs)) return rc;
    raw_len.resize(raw.size(), u->cls[ci].n);
    if (u->cls[ci].ex->kind == K_FOURSTEP) {
      // the class's L2 blocks (two phases each) rotate over the lanes, so one
      // block's passes overlap the next block's
      for (size_t r = first; r < raw.size(); r++)
        raw_lane.push_back((int)((cls_lane[ci] + (r - first) / 2) % gofft_uneven::kLanes));
    } else {
      raw_lane.resize(raw.size(), cls_lane[ci]);
    }
  }
  // order by level, keeping class order within a level; remap dependencies
  std::vector<int> order(raw.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return lvl[x] < lvl[y]; });
  std::vector<int> pos(raw.size());
  for (size_t i = 0; i < order.size(); i++) pos[order[i]] = (int)i;
  u->launch_order = pos;  // per-phase launches keep class and block order
  u->nph = (int)raw.size();
  u->ph[0].resize(u->nph);
  long long first = 0;
  for (int i = 0; i < u->nph; i++) {
    PhaseDesc p = raw[order[i]];
    if (p.dep >= 0) p.dep = pos[p.dep];
    p.first = first;
    first += p.ntiles;
    u->ph[0][i] = p;
    u->ph_level.push_back(lvl[order[i]]);
    u->ph_lane.push_back(raw_lane[order[i]]);
    u->ph_prog.push_back(progs[order[i]]);
  }
  u->total = first;
  // workspace and counters
  u->ws_bytes = wsoff;
  if (wsoff) GF_CK(cudaMalloc(&u->ws, wsoff));
  for (auto &p : u->ph[0]) {
    rebase_side(p.a.in, (char *)u->ws, &g_in_tag, &g_out_tag);
    rebase_side(p.a.out, (char *)u->ws, &g_in_tag, &g_out_tag);
    rebase_aux(p.a.aux0, (char *)u->ws, u->ws_bytes);
    rebase_aux(p.a.aux1, (char *)u->ws, u->ws_bytes);
    rebase_aux(p.a.aux2, (char *)u->ws, u->ws_bytes);
  }
  // inverse table: conjugate in on each level-0 phase, out on each last phase
  u->ph[1] = u->ph[0];
  for (int i = 0; i < u->nph; i++) {
    bool has_child = false;
    for (int j = 0; j < u->nph; j++)
      if (u->ph[0][j].dep == i) has_child = true;
    PhaseDesc &p = u->ph[1][i];
    if (p.dep < 0) p.a.cj_in = 1;
    if (!has_child) {
      p.a.cj_out = 1;
      p.a.scale = 1.0;  // set below per class length
    }
  }
  // scale 1/n on the last phase of each class (n its class length)
  for (int i = 0; i < u->nph; i++) {
    bool has_child = false;
    for (int j = 0; j < u->nph; j++)
      if (u->ph[1][j].dep == i) has_child = true;
    if (!has_child) u->ph[1][i].a.scale = 1.0 / (double)raw_len[order[i]];
  }
  // launch shape: enough threads and shared memory for every phase
  for (int i = 0; i < u->nph; i++) {
    const PhaseDesc &p = u->ph[0][i];
    const bool conv = p.op == OP_RADER || p.op == OP_BLUE;
    // an in-shared-memory Rader item runs on every thread of the CTA
    u->block = std::max(u->block, p.op == OP_RADER_IP ? 512 : p.a.lpc * p.a.lp.T);
    if (p.op == OP_RADER_IP)  // the unpadded convolution (rader_ip.cuh)
      u->smem = std::max(u->smem, (size_t)p.a.lp.n * csize(precision));
    else
      u->smem = std::max(u->smem, (size_t)p.a.lpc * spad_size(p.a.lp.n) * csize(precision) +
                                      (conv ? 2 * p.a.lpc * csize(precision) : 0));
  }
  u->block = (u->block + 31) / 32 * 32;
  const void *kp = persist_fn(precision);
  if (u->smem > 48 * 1024) GF_CK(cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)u->smem));
  int per_sm = 0, sms = 0;
  GF_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kp, u->block, u->smem));
  GF_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, u->device));
  if (per_sm < 1) return set_err(GOFFT_EUNSUPPORTED, "persistent kernel does not fit an SM");
  u->grid = (int)std::min<long long>((long long)per_sm * sms, u->total);
  for (int d = 0; d < 2; d++) GF_CK(cudaMalloc(&u->d_ph[d], u->nph * sizeof(PhaseDesc)));
  GF_CK(cudaMallocHost(&u->h_pinned, u->nph * sizeof(PhaseDesc)));
  GF_CK(cudaMalloc(&u->d_ctr, sizeof(unsigned long long) * (2 + (u->nph + 2) / 2)));
  // the counter, done counts and error word start at zero (one launch per
  // phase never writes them, and gofft_uneven_status reads the error word)
  GF_CK(cudaMemset(u->d_ctr, 0, sizeof(unsigned long long) * (2 + (u->nph + 2) / 2)));
  GF_CK(cudaEventCreateWithFlags(&u->ev_fork, cudaEventDisableTiming));
  for (int k = 1; k < gofft_uneven::kLanes; k++) {
    GF_CK(cudaStreamCreateWithFlags(&u->lane[k], cudaStreamNonBlocking));
    GF_CK(cudaEventCreateWithFlags(&u->ev_join[k], cudaEventDisableTiming));
  }
  *out = u.release();
  return GOFFT_OK;
}

extern "C" int gofft_uneven_destroy(gofft_uneven *u) {
  delete u;
  return GOFFT_OK;
}

// Writes the phase table for (in, out) when the buffers differ from the last
// call in this direction (not allowed while the stream is being captured).
static int patch(gofft_uneven *u, int dir, const void *in, void *out, cudaStream_t st) {
  if (u->last_in[dir] == in && u->last_out[dir] == out) return 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(st, &cs);
  if (cs != cudaStreamCaptureStatusNone)
    return set_err(GOFFT_EINVAL, "run the uneven batch once on these buffers before capturing it");
  std::vector<PhaseDesc> t = u->ph[dir];
  for (auto &p : t) {
    if (p.a.in.ptr == &g_in_tag) p.a.in.ptr = (void *)in;
    if (p.a.in.ptr == &g_out_tag) p.a.in.ptr = out;
    if (p.a.out.ptr == &g_out_tag) p.a.out.ptr = out;
    if (p.a.out.ptr == &g_in_tag) p.a.out.ptr = (void *)in;
  }
  if (u->extra_wait && u->nph > 1) {
    // test hook: every phase after the first waits on the first, which
    // never completes
    for (int i = 1; i < u->nph; i++) t[i].dep = 0;
    t[0].ntiles += 1;
  }
  GF_CK(cudaStreamSynchronize(st));
  GF_CK(cudaMemcpy(u->d_ph[dir], t.data(), u->nph * sizeof(PhaseDesc), cudaMemcpyHostToDevice));
  u->last_in[dir] = in;
  u->last_out[dir] = out;
  return 0;
}

extern "C" int gofft_uneven_exec(gofft_uneven *u, const void *in, void *out, int inverse, gofft_stream stream) {
  if (!u || !in || !out) return set_err(GOFFT_EINVAL, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const int dir = inverse ? 1 : 0;
  if (int rc = patch(u, dir, in, out, st)) return rc;
  if (u->persistent) {
    GF_CK(cudaMemsetAsync(u->d_ctr, 0, sizeof(unsigned long long) * (2 + (u->nph + 2) / 2), st));
    count_launch();
    const PersistFn fn = (PersistFn)persist_fn(u->prec);
    fn<<<u->grid, u->block, u->smem, st>>>(u->d_ph[dir], u->nph, u->total, u->d_ctr, done_ptr(u), err_ptr(u),
                                           u->spin_limit);
    GF_CK(cudaGetLastError());
    return GOFFT_OK;
  }
  // one launch per phase; a class's phases stay in order on its lane (its
  // dependencies are earlier phases of the same class), classes on different
  // lanes overlap; lanes fork from and join back into the caller's stream
  GF_CK(cudaEventRecord(u->ev_fork, st));
  for (int k = 1; k < gofft_uneven::kLanes; k++) GF_CK(cudaStreamWaitEvent(u->lane[k], u->ev_fork, 0));
  std::vector<PhaseDesc> t = u->ph[dir];
  int rc = 0;
  for (int r = 0; r < u->nph && !rc; r++) {
    const int i = u->launch_order[r];
    PhaseDesc p = t[i];
    if (p.a.in.ptr == &g_in_tag) p.a.in.ptr = (void *)in;
    if (p.a.out.ptr == &g_out_tag) p.a.out.ptr = out;
    const bool conv = p.op == OP_RADER || p.op == OP_BLUE;
    const cudaStream_t s = u->ph_lane[i] ? u->lane[u->ph_lane[i]] : st;
    rc = launch_line(p.op, *u->ph_prog[i], p.a, p.a.nlines, s, p.a.lpc, conv);
  }
  for (int k = 1; k < gofft_uneven::kLanes; k++) {
    cudaEventRecord(u->ev_join[k], u->lane[k]);
    cudaStreamWaitEvent(st, u->ev_join[k], 0);
  }
  if (rc) return rc;
  GF_CK(cudaGetLastError());
  return GOFFT_OK;
}

extern "C" int gofft_uneven_status(gofft_uneven *u) {
  if (!u) return set_err(GOFFT_EINVAL, "null argument");
  int err = 0;
  GF_CK(cudaDeviceSynchronize());
  GF_CK(cudaMemcpy(&err, err_ptr(u), sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return set_err(GOFFT_ETIMEOUT, "a persistent-kernel wait timed out");
  return GOFFT_OK;
}

extern "C" int gofft_uneven_set(gofft_uneven *u, int what, int64_t value) {
  if (!u) return set_err(GOFFT_EINVAL, "null argument");
  switch (what) {
    case 0: u->persistent = value ? 1 : 0; break;
    case 1: u->spin_limit = value > 0 ? value : 1; break;
    case 2:
      u->extra_wait = value ? 1 : 0;
      u->last_in[0] = u->last_in[1] = nullptr;
      u->last_out[0] = u->last_out[1] = nullptr;
      break;
    default: return set_err(GOFFT_EINVAL, "bad setting");
  }
  return GOFFT_OK;
}

extern "C" int64_t gofft_uneven_describe(const gofft_uneven *u, char *buf, int64_t cap) {
  if (!u) return -1;
  std::ostringstream o;
  o << "{\"count\":" << u->count << ",\"precision\":" << u->prec << ",\"phases\":" << u->nph
    << ",\"items\":" << u->total << ",\"grid\":" << u->grid << ",\"block\":" << u->block << ",\"smem\":" << u->smem
    << ",\"workspace\":" << u->ws_bytes << ",\"persistent\":" << u->persistent << ",\"classes\":[";
  for (size_t i = 0; i < u->cls.size(); i++)
    o << (i ? "," : "") << "{\"n\":" << u->cls[i].n << ",\"count\":" << u->cls[i].sig.size()
      << ",\"exec\":" << u->cls[i].ex->describe() << "}";
  o << "],\"phase_list\":[";
  for (int i = 0; i < u->nph; i++) {
    const PhaseDesc &p = u->ph[0][i];
    o << (i ? "," : "") << "{\"op\":" << p.op << ",\"n\":" << p.a.lp.n << ",\"lines\":" << p.a.nlines
      << ",\"lpc\":" << p.a.lpc << ",\"tiles\":" << p.ntiles << ",\"dep\":" << p.dep
      << ",\"level\":" << u->ph_level[i] << "}";
  }
  o << "]}";
  const std::string s = o.str();
  if (buf && cap > 0) {
    const size_t k = std::min<size_t>(s.size(), (size_t)cap - 1);
    memcpy(buf, s.data(), k);
    buf[k] = 0;
  }
  return (int64_t)s.size();
}
