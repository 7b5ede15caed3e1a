// api.cu -- the C-ABI (include/gofft.h): device-resident plans and the
// reference-facing entry points that mirror go-fft/fft's Go API.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <sstream>

#include "../../include/gofft.h"
#include "plan.cuh"

using namespace gf;

#define GF_CK(x)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess)                                                              \
      return set_err(GOFFT_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_));     \
  } while (0)

struct gofft_plan {
  int kind = GOFFT_C2C, prec = F64, rank = 1;
  std::vector<long long> shape;
  long long batch = 1, istride = 1, idist = 0, ostride = 1, odist = 0, total = 1;
  std::vector<std::shared_ptr<const Exec1D>> ax;  // complex exec per axis
  std::shared_ptr<const ExecReal> rx;             // real exec of the last axis (R2C)
  long long chunk = 1;                            // images per L2 block (rank-2 R2C)
  int nlanes = 1;                                 // streams the blocks rotate over (1 or kLanes)
  size_t lane_bytes = 0;                          // workspace per lane
  size_t lane_buf = 0;                            // block buffer at the start of a lane region
  long long nplane_blocks = 0;                    // complex N-D: planes per L2 block (0: unblocked)
  long long line_blocks = 0;                      // 1-D complex four-step: signals per L2 block (0: unblocked)
  cudaStream_t lane[2] = {nullptr, nullptr};      // the second lane's stream (lane[1] unused)
  cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
  size_t ws_bytes = 0;
  void *ws = nullptr;
  void *d_in = nullptr, *d_out = nullptr;
  size_t d_in_bytes = 0, d_out_bytes = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;  // host-pointer pipeline (2-D real plans)
  std::vector<cudaEvent_t> host_ev;                     // per block: inputs on the device, block transformed
  std::mutex mu;
  int device = 0;
  bool cached = false;
  ~gofft_plan() {
    if (ws) cudaFree(ws);
    if (d_in) cudaFree(d_in);
    if (d_out) cudaFree(d_out);
    for (cudaEvent_t e : host_ev) cudaEventDestroy(e);
    if (copy_in) cudaStreamDestroy(copy_in);
    if (copy_out) cudaStreamDestroy(copy_out);
    if (stream) cudaStreamDestroy(stream);
    for (int i = 0; i < 2; i++) {
      if (lane[i]) cudaStreamDestroy(lane[i]);
      if (ev_join[i]) cudaEventDestroy(ev_join[i]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
  }
};

static const char *kVersion = "gofft-b200 0.1 (sm_100a)";

extern "C" const char *gofft_last_error(void) { return last_err(); }
extern "C" const char *gofft_version(void) { return kVersion; }

// ---------------------------------------------------------------------------
// Plan construction
// ---------------------------------------------------------------------------
// Bytes of complex intermediate an L2 block of images (rank-2 real plans) or
// planes (complex N-D plans) may hold, so the row-to-column intermediate stays
// in the 126 MB L2; process-wide, read when a plan is created
// (gofft_set_l2_block_bytes).
static constexpr long long kL2BlockBytes = 48ll << 20;
static std::atomic<long long> g_l2_block_bytes{kL2BlockBytes};
static long long l2_block_bytes() { return g_l2_block_bytes.load(); }

// Items per L2 block for `units` items in at least `want` blocks: the
// smallest block count from `want` up whose equal-as-possible blocks come out
// a multiple of the lane count (when there are items for it), so every lane
// gets the same number of blocks instead of one lane running the last block
// alone.
static long long lane_chunk(long long units, long long want, int nl) {
  const long long first = (units + want - 1) / want;
  if (want <= 1) return first;
  for (long long nb = want; nb <= units; nb++) {
    const long long chunk = (units + nb - 1) / nb;
    if (((units + chunk - 1) / chunk) % nl == 0) return chunk;
  }
  return first;
}

// Lanes (streams) a blocked plan rotates its L2 blocks over, for plans created
// afterwards (gofft_set_lanes): two by default, measured best on the 2-D real
// round trip (three: 0.494-0.510 ms against 0.483 ms); one runs the blocks
// back to back on the caller's stream, so each pass is timed alone.
static constexpr int kLanes = 2;
static std::atomic<int> g_lanes{kLanes};

// Extent (elements) of `batch` lines of `len` elements at (dist, stride).
static long long extent(long long batch, long long dist, long long len, long long stride) {
  if (batch <= 0 || len <= 0) return 0;
  return (batch - 1) * dist + (len - 1) * stride + 1;
}

static int plan_ws(gofft_plan *p) {
  size_t need = 0;
  if (p->kind == GOFFT_C2C && p->line_blocks > 0) {
    // one region per lane, each for one block of signals
    p->lane_buf = 0;
    p->lane_bytes = (p->ax[0]->ws_bytes(p->line_blocks) + 255) & ~(size_t)255;
    need = (size_t)p->nlanes * p->lane_bytes;
  } else if (p->kind == GOFFT_C2C) {
    for (int a = 0; a < p->rank; a++) {
      const long long lines = (p->rank == 1 ? p->batch : p->batch * (p->total / p->shape[a]));
      need = std::max(need, p->ax[a]->ws_bytes(lines));
    }
    if (p->nplane_blocks > 0) {
      // one region per lane for the blocked last-two-axes passes
      const int r = p->rank;
      const long long kb = p->nplane_blocks;
      const size_t sub = std::max(p->ax[r - 1]->ws_bytes(kb * p->shape[r - 2]),
                                  p->ax[r - 2]->ws_bytes(kb * p->shape[r - 1]));
      p->lane_buf = 0;
      p->lane_bytes = (sub + 255) & ~(size_t)255;
      need = std::max(need, (size_t)p->nlanes * p->lane_bytes);
    }
  } else if (p->rank == 1) {
    need = p->rx->ws_bytes(p->batch);
  } else {
    // per lane: the block's spectrum buffer, then the passes' own workspace
    const long long rows = p->shape[0], rc = p->shape[1] / 2 + 1;
    // the tiled intermediate rounds the block's column-lines up to a whole group
    const long long W = 64 / (long long)csize(p->prec);
    const size_t cols_buf = ((size_t)rows * (rc * p->chunk + W - 1) * csize(p->prec) + 255) & ~(size_t)255;
    const size_t sub = std::max(p->rx->ws_bytes(rows * p->chunk), p->ax[0]->ws_bytes(rc * p->chunk));
    p->lane_buf = cols_buf;
    p->lane_bytes = (cols_buf + sub + 255) & ~(size_t)255;
    need = p->lane_bytes * p->nlanes;
  }
  p->ws_bytes = need;
  if (need) {
    cudaError_t e = cudaMalloc(&p->ws, need);
    if (e != cudaSuccess) return set_err(GOFFT_ENOMEM, std::string("workspace: ") + cudaGetErrorString(e));
  }
  return 0;
}

extern "C" int gofft_plan_create(int kind, int precision, const int64_t *shape, int rank,
                                 int64_t batch, int64_t istride, int64_t idist, int64_t ostride,
                                 int64_t odist, gofft_plan **out) {
  if (!out) return set_err(GOFFT_EINVAL, "null output handle");
  *out = nullptr;
  if (kind != GOFFT_C2C && kind != GOFFT_R2C) return set_err(GOFFT_EINVAL, "bad kind");
  if (precision < 0 || precision > 2) return set_err(GOFFT_EINVAL, "bad precision");
  if (rank < 1 || rank > 16 || !shape) return set_err(GOFFT_EINVAL, "rank must be in [1,16]");
  if (batch < 1) return set_err(GOFFT_EINVAL, "batch must be >= 1");
  for (int a = 0; a < rank; a++)
    if (shape[a] <= 0) return set_err(GOFFT_EINVAL, "fft: shape lengths must be positive");
  if (kind == GOFFT_R2C && rank > 2) return set_err(GOFFT_EUNSUPPORTED, "real transforms support rank 1 and 2");
  std::unique_ptr<gofft_plan> p(new gofft_plan());
  p->kind = kind;
  p->prec = precision;
  p->rank = rank;
  p->batch = batch;
  cudaGetDevice(&p->device);
  p->shape.assign(shape, shape + rank);
  p->total = 1;
  for (long long s : p->shape) p->total *= s;
  const long long last = p->shape[rank - 1];
  const long long rc = last / 2 + 1;
  const long long in_line = kind == GOFFT_C2C ? p->total : p->total;            // reals or complex
  const long long out_line = kind == GOFFT_C2C ? p->total : p->total / last * rc;  // bins
  p->istride = istride > 0 ? istride : 1;
  p->ostride = ostride > 0 ? ostride : 1;
  p->idist = idist > 0 ? idist : in_line * p->istride;
  p->odist = odist > 0 ? odist : out_line * p->ostride;
  if (rank > 1 && (p->istride != 1 || p->ostride != 1))
    return set_err(GOFFT_EUNSUPPORTED, "rank > 1 needs unit element strides");
  if (kind == GOFFT_C2C) {
    for (int a = 0; a < rank; a++) {
      auto ex = get_exec(p->shape[a], precision);
      if (!ex) return GOFFT_ECUDA;
      p->ax.push_back(ex);
    }
    if (rank == 1 && p->ax[0]->kind == K_FOURSTEP) {
      // four-step signals per L2 block: a block's pass-1 output stays in L2
      // for pass 2; blocks alternate lanes, so one block's passes overlap
      // the next block's
      const long long per = p->shape[0] * (long long)csize(precision);
      const long long cmax = std::max<long long>(1, std::min<long long>(batch, l2_block_bytes() / per));
      const long long nblocks = (batch + cmax - 1) / cmax;
      if (nblocks > 1 && g_lanes.load() > 1) {
        p->nlanes = g_lanes.load();
        p->line_blocks = lane_chunk(batch, nblocks, p->nlanes);
      }
    }
    if (rank >= 2 && p->shape[rank - 1] > 1 && p->shape[rank - 2] > 1) {
      // planes (the last two axes) per L2 block: both axes run while a
      // block's planes sit in L2, on two lanes; leading axes run afterwards
      const long long plane = p->shape[rank - 1] * p->shape[rank - 2];
      const bool merged = p->idist == p->total && p->odist == p->total;
      const long long units = (merged ? batch : 1) * (p->total / plane);
      const long long budget = l2_block_bytes();
      const long long cmax =
          std::max<long long>(1, std::min<long long>(units, budget / (plane * (long long)csize(precision))));
      const long long nblocks = (units + cmax - 1) / cmax;
      if (nblocks > 1 && g_lanes.load() > 1) {
        p->nlanes = g_lanes.load();
        p->nplane_blocks = lane_chunk(units, nblocks, p->nlanes);
      }
    }
  } else {
    p->rx = get_real(last, precision);
    if (!p->rx) return GOFFT_ECUDA;
    if (rank == 2) {
      auto ex = get_exec(p->shape[0], precision);
      if (!ex) return GOFFT_ECUDA;
      p->ax.push_back(ex);
      if (p->istride != 1 || p->idist != p->total || p->ostride != 1 || p->odist != p->shape[0] * rc)
        return set_err(GOFFT_EUNSUPPORTED, "2-D real transforms need contiguous images");
      // images per block: keep a block's complex intermediate L2-resident
      const long long budget = l2_block_bytes();
      const long long per = p->shape[0] * rc * (long long)csize(precision);
      const long long cmax = std::max<long long>(1, std::min<long long>(batch, budget / std::max<long long>(1, per)));
      // at least two blocks when there are two images, so the lanes overlap
      // one block's row passes with the other block's column pass even when
      // the whole batch would fit one L2 block
      const long long nblocks = std::max<long long>((batch + cmax - 1) / cmax, batch >= 2 ? 2 : 1);
      // lanes: block i+1's passes overlap block i's (each pass alone ramps
      // up and drains; the other lanes fill those gaps)
      const bool lanes = nblocks > 1 && g_lanes.load() > 1;
      if (lanes) p->nlanes = g_lanes.load();
      p->chunk = lanes ? lane_chunk(batch, nblocks, p->nlanes) : (batch + nblocks - 1) / nblocks;  // balanced blocks
    }
  }
  if (int rc2 = plan_ws(p.get())) return rc2;
  if (p->nlanes > 1) {
    GF_CK(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
    for (int i = 0; i + 1 < p->nlanes; i++) {
      GF_CK(cudaStreamCreateWithFlags(&p->lane[i], cudaStreamNonBlocking));
      GF_CK(cudaEventCreateWithFlags(&p->ev_join[i], cudaEventDisableTiming));
    }
  }
  *out = p.release();
  return GOFFT_OK;
}

extern "C" int gofft_plan_destroy(gofft_plan *p) {
  if (!p) return GOFFT_OK;
  if (p->cached) return GOFFT_OK;  // memoised plans live for the process
  delete p;
  return GOFFT_OK;
}

extern "C" int gofft_plan_workspace_size(const gofft_plan *p, size_t *bytes) {
  if (!p || !bytes) return set_err(GOFFT_EINVAL, "null argument");
  *bytes = p->ws_bytes;
  return GOFFT_OK;
}

extern "C" int64_t gofft_plan_describe(const gofft_plan *p, char *buf, int64_t cap) {
  if (!p) return -1;
  std::ostringstream o;
  o << "{\"kind\":\"" << (p->kind == GOFFT_C2C ? "c2c" : "r2c") << "\",\"precision\":" << p->prec
    << ",\"batch\":" << p->batch << ",\"shape\":[";
  for (int a = 0; a < p->rank; a++) o << (a ? "," : "") << p->shape[a];
  o << "],\"workspace\":" << p->ws_bytes << ",\"chunk\":" << p->chunk << ",\"line_blocks\":" << p->line_blocks
    << ",\"axes\":[";
  for (size_t a = 0; a < p->ax.size(); a++) o << (a ? "," : "") << p->ax[a]->describe();
  o << "]";
  if (p->rx) o << ",\"real\":" << p->rx->describe();
  o << "}";
  const std::string s = o.str();
  if (buf && cap > 0) {
    const size_t k = std::min<size_t>(s.size(), (size_t)cap - 1);
    memcpy(buf, s.data(), k);
    buf[k] = 0;
  }
  return (int64_t)s.size();
}

extern "C" int64_t gofft_plan_table(const gofft_plan *p, int which, int64_t *out, int64_t cap) {
  if (!p || p->kind != GOFFT_C2C || p->rank != 1) return -1;
  const Exec1D &e = *p->ax[0];
  std::vector<int64_t> v;
  if ((which == 0 || which == 1) && e.kind == K_RADER) {
    std::vector<int> t(e.n - 1);
    if (cudaMemcpy(t.data(), which == 0 ? e.perm : e.iperm, t.size() * sizeof(int),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      return -1;
    v.assign(t.begin(), t.end());
  } else if (which == 2 && e.kind == K_BLUE) {
    v.resize(e.n);
    if (cudaMemcpy(v.data(), e.jj, v.size() * sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess)
      return -1;
  } else if (which == 3 && e.kind == K_RADER) {
    v = {e.g, e.cl};
  } else if (which == 4 && e.kind == K_BLUE) {
    v = {e.m};
  } else {
    return -1;
  }
  if (out)
    for (int64_t i = 0; i < (int64_t)v.size() && i < cap; i++) out[i] = v[i];
  return (int64_t)v.size();
}

// ---------------------------------------------------------------------------
// Execution on device pointers
// ---------------------------------------------------------------------------
// The L2 blocks of a plan (images of a rank-2 real plan, planes of a complex
// N-D plan) rotate over the caller's stream and the plan's lane streams
// (forked from and joined back into the caller's stream), each lane with its
// own workspace region: the block buffer (real plans), then the passes'
// workspace.
struct Lanes {
  gofft_plan *p;
  cudaStream_t st;
  int n = 1;  // lanes in use
  Lanes(gofft_plan *p_, cudaStream_t st_) : p(p_), st(st_) {}
  int fork(long long nblocks) {
    n = nblocks > 1 ? (int)std::min<long long>(p->nlanes, nblocks) : 1;
    if (n == 1) return 0;
    GF_CK(cudaEventRecord(p->ev_fork, st));
    for (int i = 0; i + 1 < n; i++) GF_CK(cudaStreamWaitEvent(p->lane[i], p->ev_fork, 0));
    return 0;
  }
  int lane_of(long long blk) const { return n > 1 ? (int)(blk % n) : 0; }
  cudaStream_t stream(long long blk) const {
    const int k = lane_of(blk);
    return k ? p->lane[k - 1] : st;
  }
  char *buf(long long blk) const { return (char *)p->ws + (size_t)lane_of(blk) * p->lane_bytes; }
  char *sub(long long blk) const { return buf(blk) + p->lane_buf; }
  // Joins the lanes back into the caller's stream; keeps the first error.
  int join(int rc) {
    if (n == 1) return rc;
    cudaError_t err = cudaSuccess;
    for (int i = 0; i + 1 < n; i++) {
      cudaError_t e1 = cudaEventRecord(p->ev_join[i], p->lane[i]);
      cudaError_t e2 = cudaStreamWaitEvent(st, p->ev_join[i], 0);
      if (err == cudaSuccess) err = e1 != cudaSuccess ? e1 : e2;
    }
    n = 1;
    if (rc) return rc;
    if (err != cudaSuccess) return set_err(GOFFT_ECUDA, std::string("lane join: ") + cudaGetErrorString(err));
    return 0;
  }
};

// cj: transform direction (1 = inverse, as conj(FFT(conj .))); scaled: apply
// the inverse's 1/n per axis.  The plain transforms have cj == scaled; the
// adjoints flip the direction and keep the scaling.
static int exec_c2c_dir(gofft_plan *p, const void *in, void *out, int cj, int scaled, cudaStream_t st) {
  if (p->rank == 1 && p->line_blocks > 0) {
    const double sc = scaled ? 1.0 / (double)p->shape[0] : 1.0;
    const size_t c = csize(p->prec);
    const long long kb0 = p->line_blocks;
    Lanes ln(p, st);
    if (int e = ln.fork((p->batch + kb0 - 1) / kb0)) return e;
    long long blk = 0;
    for (long long b0 = 0; b0 < p->batch; b0 += kb0, blk++) {
      const long long kb = std::min(kb0, p->batch - b0);
      const Side si = mk_side((char *)in + (size_t)b0 * p->idist * c, p->idist, 0, p->istride, 1);
      const Side so = mk_side((char *)out + (size_t)b0 * p->odist * c, p->odist, 0, p->ostride, 1);
      if (int e = p->ax[0]->exec(si, so, kb, cj, cj, sc, ln.sub(blk), ln.stream(blk))) return ln.join(e);
    }
    return ln.join(GOFFT_OK);
  }
  if (p->rank == 1) {
    const double sc = scaled ? 1.0 / (double)p->shape[0] : 1.0;
    return p->ax[0]->exec(mk_side((void *)in, p->idist, 0, p->istride, 1),
                          mk_side(out, p->odist, 0, p->ostride, 1), p->batch, cj, cj, sc, p->ws, st);
  }
  const size_t c = csize(p->prec);
  const bool merged = p->idist == p->total && p->odist == p->total;
  const long long nb = merged ? 1 : p->batch;
  const long long per = merged ? p->batch : 1;
  const int r = p->rank;
  for (long long b = 0; b < nb; b++) {
    const char *src = (const char *)in + (size_t)b * p->idist * c;
    char *dst = (char *)out + (size_t)b * p->odist * c;
    bool first = true;
    int lead = r;  // axes 0..lead-1 still to run over the whole array
    if (p->nplane_blocks > 0) {
      // the last two axes per L2 block of planes, blocks alternating lanes
      const long long Lr = p->shape[r - 1], Lc = p->shape[r - 2], plane = Lr * Lc;
      const long long units = per * (p->total / plane), kb0 = p->nplane_blocks;
      Lanes ln(p, st);
      if (int e = ln.fork((units + kb0 - 1) / kb0)) return e;
      long long blk = 0;
      for (long long k0 = 0; k0 < units; k0 += kb0, blk++) {
        const long long kb = std::min(kb0, units - k0);
        const size_t off = (size_t)k0 * plane * c;
        const cudaStream_t s = ln.stream(blk);
        char *wsx = ln.sub(blk);
        const Side rin = mk_side((void *)(src + off), Lr, 1, 1, 1), rout = mk_side(dst + off, Lr, 1, 1, 1);
        if (int e = p->ax[r - 1]->exec(rin, rout, kb * Lc, cj, cj, scaled ? 1.0 / (double)Lr : 1.0, wsx, s))
          return ln.join(e);
        const Side cs = mk_side(dst + off, plane, 1, Lr, Lr);
        if (int e = p->ax[r - 2]->exec(cs, cs, kb * Lr, cj, cj, scaled ? 1.0 / (double)Lc : 1.0, wsx, s))
          return ln.join(e);
      }
      if (int e = ln.join(GOFFT_OK)) return e;
      first = false;
      lead = r - 2;
    }
    long long inner = p->total;
    for (int a = 0; a < lead; a++) {
      const long long L = p->shape[a];
      inner /= L;
      if (L == 1) continue;
      const Side sd_in = mk_side(first ? (void *)src : (void *)dst, L * inner, 1, inner, inner);
      const Side sd_out = mk_side(dst, L * inner, 1, inner, inner);
      const long long lines = per * (p->total / L);
      const double sc = scaled ? 1.0 / (double)L : 1.0;
      if (int rc = p->ax[a]->exec(sd_in, sd_out, lines, cj, cj, sc, p->ws, st)) return rc;
      first = false;
    }
    if (first && src != dst) GF_CK(cudaMemcpyAsync(dst, src, (size_t)per * p->total * c, cudaMemcpyDeviceToDevice, st));
  }
  return GOFFT_OK;
}

static int exec_c2c(gofft_plan *p, const void *in, void *out, int inverse, cudaStream_t st) {
  return exec_c2c_dir(p, in, out, inverse ? 1 : 0, inverse ? 1 : 0, st);
}


// Whether a rank-2 real plan keeps its row-to-column intermediate in the
// tiled layout (TiledPos in ops.cuh): groups of W column-lines (64 bytes of
// a row: 4 complex128 or 8 complex64), each a contiguous rows x W block, so
// the column pass reads or writes whole contiguous tiles on that side
// instead of one 64-byte row segment per row.  FP64 plans only: the FP32
// forms measured slower tiled (32 x 1024^2 round trip 0.2664 ms image layout,
// 0.2718 ms tiled, 0.2685 ms tiled forward only; their row passes lose more
// than the column pass gains).  Packed fused row transforms only (even row
// length, one CTA per row), and not while the opt-in TMA-fed kernel is on (it
// reads and writes the image layout).
static bool tiled_real2(const gofft_plan *p) {
  return p->prec == F64 && p->rank == 2 && p->shape[0] > 1 && p->rx->can_tile() && !tma_pipeline();
}

// The column pass's view of the tiled intermediate: line L (image * rc +
// column) starts at (L / W) * W * rows + L % W, elements W apart.
static Side tiled_side(const gofft_plan *p, char *buf) {
  const long long W = 64 / (long long)csize(p->prec), rows = p->shape[0];
  return mk_side(buf, W * rows, 1, W, W);
}

// One block of nb images of a rank-2 real forward, on stream s: rows into the
// lane's block buffer colbuf (tiled), columns from there into dst; wsx is the
// lane's pass workspace.
static int r2c_block(gofft_plan *p, const char *src, char *dst, long long nb, char *colbuf, char *wsx,
                     cudaStream_t s, double wsc) {
  const long long rows = p->shape[0], cols = p->shape[1], rc = cols / 2 + 1;
  const Side cs = mk_side(dst, rows * rc, 1, rc, rc);
  if (tiled_real2(p)) {
    // rows: real transform along the last axis (rfft2.go:41-51)
    if (int e = p->rx->r2c(contig((void *)src, cols), contig(colbuf, rc), nb * rows, wsx, s, wsc, rows)) return e;
    // columns: complex transform down each of the rc columns (rfft2.go:53-72)
    return p->ax[0]->exec(tiled_side(p, colbuf), cs, nb * rc, 0, 0, 1.0, wsx, s);
  }
  if (int e = p->rx->r2c(contig((void *)src, cols), contig(dst, rc), nb * rows, wsx, s, wsc)) return e;
  if (rows > 1) {
    if (int e = p->ax[0]->exec(cs, cs, nb * rc, 0, 0, 1.0, wsx, s)) return e;
  }
  return GOFFT_OK;
}

// One block of nb images of a rank-2 real inverse: columns into the lane's
// block buffer colbuf (tiled when the plan allows), then the real rows into
// dst.
static int c2r_block(gofft_plan *p, const char *src, char *dst, long long nb, char *colbuf, char *wsx,
                     cudaStream_t s, bool adj) {
  const long long rows = p->shape[0], cols = p->shape[1], rc = cols / 2 + 1;
  const bool tiled = tiled_real2(p);
  // columns: complex inverse, normalised by 1/rows (rfft2.go:100-120)
  const Side cin = mk_side((void *)src, rows * rc, 1, rc, rc);
  const Side cout = tiled ? tiled_side(p, colbuf) : mk_side(colbuf, rows * rc, 1, rc, rc);
  if (int e = p->ax[0]->exec(cin, cout, nb * rc, 1, 1, adj ? 1.0 : 1.0 / (double)rows, wsx, s)) return e;
  // rows: real inverse of length cols (rfft2.go:122-136)
  return p->rx->c2r(contig(colbuf, rc), (int)rc, contig(dst, cols), nb * rows, adj ? (double)cols : 1.0, wsx, s,
                    adj, tiled ? rows : 0);
}

// wsc != 0: the adjoint of the inverse (edge-bin weighting with scale wsc on
// the row pass, the only real one).
static int exec_r2c(gofft_plan *p, const void *in, void *out, cudaStream_t st, double wsc = 0.0) {
  if (p->rank == 1) {
    return p->rx->r2c(mk_side((void *)in, p->idist, 0, p->istride, 1), mk_side(out, p->odist, 0, p->ostride, 1),
                      p->batch, p->ws, st, wsc);
  }
  const long long rows = p->shape[0], cols = p->shape[1], rc = cols / 2 + 1;
  const size_t r = rsize(p->prec), c = csize(p->prec);
  Lanes ln(p, st);
  if (int e = ln.fork((p->batch + p->chunk - 1) / p->chunk)) return e;
  long long blk = 0;
  for (long long b0 = 0; b0 < p->batch; b0 += p->chunk, blk++) {
    const long long nb = std::min(p->chunk, p->batch - b0);
    const char *src = (const char *)in + (size_t)b0 * rows * cols * r;
    char *dst = (char *)out + (size_t)b0 * rows * rc * c;
    if (int e = r2c_block(p, src, dst, nb, ln.buf(blk), ln.sub(blk), ln.stream(blk), wsc)) return ln.join(e);
  }
  return ln.join(GOFFT_OK);
}

// adj: the adjoint of the forward -- unnormalised, interior bins halved.
static int exec_c2r(gofft_plan *p, const void *in, long long nbins, void *out, cudaStream_t st,
                    bool adj = false) {
  const long long last = p->shape[p->rank - 1], rc = last / 2 + 1;
  if (nbins <= 0 || nbins > rc) nbins = rc;
  if (p->rank == 1) {
    // bins on the plan's complex side (odist/ostride), reals on its real side
    return p->rx->c2r(mk_side((void *)in, p->odist, 0, p->ostride, 1), (int)nbins,
                      mk_side(out, p->idist, 0, p->istride, 1), p->batch, adj ? (double)last : 1.0, p->ws, st,
                      adj);
  }
  // 2-D: in (complex) is the plan's output side; out (real) its input side
  const long long rows = p->shape[0], cols = last;
  const size_t r = rsize(p->prec), c = csize(p->prec);
  Lanes ln(p, st);
  if (int e = ln.fork((p->batch + p->chunk - 1) / p->chunk)) return e;
  long long blk = 0;
  for (long long b0 = 0; b0 < p->batch; b0 += p->chunk, blk++) {
    const long long nb = std::min(p->chunk, p->batch - b0);
    const char *src = (const char *)in + (size_t)b0 * rows * rc * c;
    char *dst = (char *)out + (size_t)b0 * rows * cols * r;
    if (int e = c2r_block(p, src, dst, nb, ln.buf(blk), ln.sub(blk), ln.stream(blk), adj)) return ln.join(e);
  }
  return ln.join(GOFFT_OK);
}

extern "C" int gofft_exec_c2c(gofft_plan *p, const void *in, void *out, int inverse, gofft_stream stream) {
  if (!p || !in || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_C2C) return set_err(GOFFT_EINVAL, "plan is not complex-to-complex");
  return exec_c2c(p, in, out, inverse, (cudaStream_t)stream);
}
extern "C" int gofft_exec_r2c(gofft_plan *p, const void *in, void *out, gofft_stream stream) {
  if (!p || !in || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_R2C) return set_err(GOFFT_EINVAL, "plan is not real");
  return exec_r2c(p, in, out, (cudaStream_t)stream);
}
extern "C" int gofft_exec_c2r(gofft_plan *p, const void *in, int64_t nbins, void *out, gofft_stream stream) {
  if (!p || !in || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_R2C) return set_err(GOFFT_EINVAL, "plan is not real");
  return exec_c2r(p, in, nbins, out, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Host-pointer execution
// ---------------------------------------------------------------------------
// The plan's own stream for the host-pointer calls, created by the first
// such call (under the plan's lock): plans used only on device pointers never
// create one, which keeps plan construction short.
static int ensure_stream(gofft_plan *p) {
  if (!p->stream) GF_CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  return 0;
}

static int ensure_staging(gofft_plan *p, size_t in_b, size_t out_b) {
  if (int rc = ensure_stream(p)) return rc;
  if (p->d_in_bytes < in_b) {
    if (p->d_in) cudaFree(p->d_in);
    p->d_in = nullptr;
    p->d_in_bytes = 0;
    cudaError_t e = cudaMalloc(&p->d_in, in_b);
    if (e != cudaSuccess) return set_err(GOFFT_ENOMEM, "staging buffer");
    p->d_in_bytes = in_b;
  }
  if (p->d_out_bytes < out_b) {
    if (p->d_out) cudaFree(p->d_out);
    p->d_out = nullptr;
    p->d_out_bytes = 0;
    cudaError_t e = cudaMalloc(&p->d_out, out_b);
    if (e != cudaSuccess) return set_err(GOFFT_ENOMEM, "staging buffer");
    p->d_out_bytes = out_b;
  }
  return 0;
}

static size_t c2c_bytes(const gofft_plan *p, bool in) {
  const long long d = in ? p->idist : p->odist, s = in ? p->istride : p->ostride;
  const long long el = p->rank == 1 ? extent(p->batch, d, p->total, s) : (p->batch - 1) * d + p->total;
  return (size_t)el * csize(p->prec);
}
static size_t real_bytes(const gofft_plan *p) {
  const long long el = p->rank == 1 ? extent(p->batch, p->idist, p->total, p->istride) : p->batch * p->total;
  return (size_t)el * rsize(p->prec);
}
static size_t bins_bytes(const gofft_plan *p) {
  const long long rc = p->shape[p->rank - 1] / 2 + 1;
  const long long el = p->rank == 1 ? extent(p->batch, p->odist, rc, p->ostride)
                                    : p->batch * (p->total / p->shape[p->rank - 1]) * rc;
  return (size_t)el * csize(p->prec);
}

static int host_run(gofft_plan *p, const void *in, size_t in_b, void *out, size_t out_b, int which,
                    int inverse, long long nbins) {
  std::lock_guard<std::mutex> lk(p->mu);
  if (int rc = ensure_staging(p, in_b, out_b)) return rc;
  GF_CK(cudaMemcpyAsync(p->d_in, in, in_b, cudaMemcpyHostToDevice, p->stream));
  int rc = 0;
  if (which == 0) rc = exec_c2c(p, p->d_in, p->d_out, inverse, p->stream);
  else if (which == 1) rc = exec_r2c(p, p->d_in, p->d_out, p->stream);
  else rc = exec_c2r(p, p->d_in, nbins, p->d_out, p->stream);
  if (rc) return rc;
  GF_CK(cudaMemcpyAsync(out, p->d_out, out_b, cudaMemcpyDeviceToHost, p->stream));
  GF_CK(cudaStreamSynchronize(p->stream));
  return GOFFT_OK;
}

// Host-pointer execution of a rank-2 real plan, pipelined per block of
// images: the host-to-device copy of block k+1 (copy-in stream), the
// transforms of block k (on the block's lane) and the device-to-host copy of
// block k-1 (copy-out stream) run at once, so both PCIe directions and the
// GPU work together.  Blocks are half an L2 block and never fewer than two
// images (the configuration measured and tested; one-image blocks are not
// used), which keeps the pipeline's fill and drain short.  which: 1 forward,
// 2 inverse.
static long long host_block_images(const gofft_plan *p) { return std::max<long long>(2, p->chunk / 2); }

static bool host_ranges_overlap(const void *a, size_t na, const void *b, size_t nb) {
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return x < y + nb && y < x + na;
}

static int host_run_real2(gofft_plan *p, const void *in, void *out, int which) {
  const long long rows = p->shape[0], cols = p->shape[1], rc = cols / 2 + 1;
  const size_t rimg = (size_t)rows * cols * rsize(p->prec), cimg = (size_t)rows * rc * csize(p->prec);
  const size_t in_img = which == 1 ? rimg : cimg, out_img = which == 1 ? cimg : rimg;
  const long long hb = host_block_images(p);
  const long long nblk = (p->batch + hb - 1) / hb;
  std::lock_guard<std::mutex> lk(p->mu);
  if (int e = ensure_staging(p, in_img * p->batch, out_img * p->batch)) return e;
  if (!p->copy_in) GF_CK(cudaStreamCreateWithFlags(&p->copy_in, cudaStreamNonBlocking));
  if (!p->copy_out) GF_CK(cudaStreamCreateWithFlags(&p->copy_out, cudaStreamNonBlocking));
  while ((long long)p->host_ev.size() < 2 * nblk) {
    cudaEvent_t e;
    GF_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    p->host_ev.push_back(e);
  }
  const int nl = std::max(1, p->nlanes);
  int rc_ = GOFFT_OK;
  long long blk = 0;
  for (long long b0 = 0; b0 < p->batch && rc_ == GOFFT_OK; b0 += hb, blk++) {
    const long long nb = std::min(hb, p->batch - b0);
    char *din = (char *)p->d_in + (size_t)b0 * in_img, *dout = (char *)p->d_out + (size_t)b0 * out_img;
    cudaEvent_t ready = p->host_ev[2 * blk], done = p->host_ev[2 * blk + 1];
    const int k = (int)(blk % nl);
    const cudaStream_t s = k ? p->lane[k - 1] : p->stream;
    char *buf = (char *)p->ws + (size_t)k * p->lane_bytes;
    cudaError_t ce = cudaMemcpyAsync(din, (const char *)in + (size_t)b0 * in_img, (size_t)nb * in_img,
                                     cudaMemcpyHostToDevice, p->copy_in);
    if (ce == cudaSuccess) ce = cudaEventRecord(ready, p->copy_in);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s, ready, 0);
    if (ce != cudaSuccess) {
      rc_ = set_err(GOFFT_ECUDA, std::string("host pipeline: ") + cudaGetErrorString(ce));
      break;
    }
    rc_ = which == 1 ? r2c_block(p, din, dout, nb, buf, buf + p->lane_buf, s, 0.0)
                     : c2r_block(p, din, dout, nb, buf, buf + p->lane_buf, s, false);
    if (rc_) break;
    ce = cudaEventRecord(done, s);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(p->copy_out, done, 0);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync((char *)out + (size_t)b0 * out_img, dout, (size_t)nb * out_img, cudaMemcpyDeviceToHost,
                           p->copy_out);
    if (ce != cudaSuccess) rc_ = set_err(GOFFT_ECUDA, std::string("host pipeline: ") + cudaGetErrorString(ce));
  }
  // every stream drains before returning, on success and on error alike
  cudaError_t e1 = cudaStreamSynchronize(p->copy_in);
  cudaError_t e2 = cudaStreamSynchronize(p->stream);
  cudaError_t e3 = nl > 1 ? cudaStreamSynchronize(p->lane[0]) : cudaSuccess;
  cudaError_t e5 = nl > 2 ? cudaStreamSynchronize(p->lane[1]) : cudaSuccess;
  cudaError_t e4 = cudaStreamSynchronize(p->copy_out);
  if (rc_) return rc_;
  for (cudaError_t e : {e1, e2, e3, e5, e4})
    if (e != cudaSuccess) return set_err(GOFFT_ECUDA, std::string("host pipeline: ") + cudaGetErrorString(e));
  return GOFFT_OK;
}

// The pipelined path applies to 2-D real plans with at least two blocks of
// images and host buffers that do not overlap (an aliased output would
// overwrite inputs not yet copied).  A host block runs through one lane's
// workspace, which holds `chunk` images (one L2 block): plans whose host
// block would be larger (chunk < 2, i.e. one image's spectrum fills more than
// half the L2 block budget) take the serial path instead.
static bool use_real2_pipeline(const gofft_plan *p, const void *in, size_t in_b, const void *out, size_t out_b) {
  return p->rank == 2 && host_block_images(p) <= p->chunk && p->batch >= 2 * host_block_images(p) &&
         !host_ranges_overlap(in, in_b, out, out_b);
}

extern "C" int gofft_exec_c2c_host(gofft_plan *p, const void *in, void *out, int inverse) {
  if (!p || !in || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_C2C) return set_err(GOFFT_EINVAL, "plan is not complex-to-complex");
  return host_run(p, in, c2c_bytes(p, true), out, c2c_bytes(p, false), 0, inverse, 0);
}
extern "C" int gofft_exec_r2c_host(gofft_plan *p, const void *in, void *out) {
  if (!p || !in || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_R2C) return set_err(GOFFT_EINVAL, "plan is not real");
  if (use_real2_pipeline(p, in, real_bytes(p), out, bins_bytes(p))) return host_run_real2(p, in, out, 1);
  return host_run(p, in, real_bytes(p), out, bins_bytes(p), 1, 0, 0);
}
extern "C" int gofft_exec_c2r_host(gofft_plan *p, const void *in, int64_t nbins, void *out) {
  if (!p || !in || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_R2C) return set_err(GOFFT_EINVAL, "plan is not real");
  if (use_real2_pipeline(p, in, bins_bytes(p), out, real_bytes(p))) return host_run_real2(p, in, out, 2);
  return host_run(p, in, bins_bytes(p), out, real_bytes(p), 2, 0, nbins);
}

// ---------------------------------------------------------------------------
// Reference-facing entry points (FP64, host buffers)
// ---------------------------------------------------------------------------
static gofft_plan *make_1d(int kind, long long n) {
  gofft_plan *p = nullptr;
  const int64_t sh[1] = {n};
  if (gofft_plan_create(kind, GOFFT_F64, sh, 1, 1, 1, 0, 1, 0, &p) != GOFFT_OK) return nullptr;
  return p;
}

extern "C" int gofft_new_plan(int64_t n, gofft_plan **out) {
  if (!out) return set_err(GOFFT_EINVAL, "null output handle");
  if (n < 0) return set_err(GOFFT_EINVAL, "fft: negative length");
  gofft_plan *p = nullptr;
  if (n == 0) {
    p = new gofft_plan();
    p->shape = {0};
    p->total = 0;
  } else {
    p = make_1d(GOFFT_C2C, n);
    if (!p) return GOFFT_ECUDA;
  }
  *out = p;
  return GOFFT_OK;
}

// Memoised plans keyed by length (plan.go:283-317 / rfft.go:48-64): built
// outside the lock, first store wins.
static gofft_plan *memo(std::map<long long, gofft_plan *> &m, std::mutex &mu, long long n, bool real) {
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = m.find(n);
    if (it != m.end()) return it->second;
  }
  gofft_plan *p = nullptr;
  if (real) {
    p = make_1d(GOFFT_R2C, n);
  } else if (gofft_new_plan(n, &p) != GOFFT_OK) {
    p = nullptr;
  }
  if (!p) return nullptr;
  p->cached = true;
  std::lock_guard<std::mutex> lk(mu);
  auto it = m.find(n);
  if (it != m.end()) {
    p->cached = false;
    delete p;
    return it->second;
  }
  m[n] = p;
  return p;
}
static std::mutex g_cmu, g_rmu;
static std::map<long long, gofft_plan *> g_cplans, g_rplans;

extern "C" int gofft_cached_plan(int64_t n, gofft_plan **out) {
  if (!out) return set_err(GOFFT_EINVAL, "null output handle");
  if (n < 0) return set_err(GOFFT_EINVAL, "fft: negative length");
  *out = memo(g_cplans, g_cmu, n, false);
  return *out ? GOFFT_OK : GOFFT_ECUDA;
}

extern "C" int64_t gofft_plan_len(const gofft_plan *p) { return p ? (p->shape.empty() ? 0 : p->shape.back()) : 0; }

static int plan_c2c_host(gofft_plan *p, double *dst, const double *src, int inverse) {
  if (!p || (!dst && p->total) || (!src && p->total)) return set_err(GOFFT_EINVAL, "null argument");
  if (p->total == 0) return GOFFT_OK;
  if (p->kind != GOFFT_C2C || p->rank != 1 || p->batch != 1) return set_err(GOFFT_EINVAL, "not a 1-D complex plan");
  return gofft_exec_c2c_host(p, src, dst, inverse);
}
extern "C" int gofft_plan_fft(gofft_plan *p, double *dst, const double *src) { return plan_c2c_host(p, dst, src, 0); }
extern "C" int gofft_plan_ifft(gofft_plan *p, double *dst, const double *src) { return plan_c2c_host(p, dst, src, 1); }

extern "C" int gofft_new_real_plan(int64_t n, gofft_plan **out) {
  if (!out) return set_err(GOFFT_EINVAL, "null output handle");
  if (n < 0) return set_err(GOFFT_EINVAL, "fft: negative length");
  gofft_plan *p = nullptr;
  if (n == 0) {
    p = new gofft_plan();
    p->kind = GOFFT_R2C;
    p->shape = {0};
    p->total = 0;
  } else {
    p = make_1d(GOFFT_R2C, n);
    if (!p) return GOFFT_ECUDA;
  }
  *out = p;
  return GOFFT_OK;
}

extern "C" int gofft_real_plan_rfft(gofft_plan *p, double *dst, const double *src) {
  if (!p) return set_err(GOFFT_EINVAL, "null plan");
  if (p->total == 0) return GOFFT_OK;
  if (p->kind != GOFFT_R2C || p->rank != 1 || p->batch != 1) return set_err(GOFFT_EINVAL, "not a 1-D real plan");
  if (!dst || !src) return set_err(GOFFT_EINVAL, "null argument");
  return gofft_exec_r2c_host(p, src, dst);
}

extern "C" int gofft_real_plan_irfft(gofft_plan *p, double *dst, const double *src, int64_t nsrc) {
  if (!p) return set_err(GOFFT_EINVAL, "null plan");
  if (p->total == 0) return GOFFT_OK;
  if (p->kind != GOFFT_R2C || p->rank != 1 || p->batch != 1) return set_err(GOFFT_EINVAL, "not a 1-D real plan");
  if (!dst) return set_err(GOFFT_EINVAL, "null argument");
  const long long rc = p->total / 2 + 1;
  long long nb = std::min<long long>(std::max<long long>(nsrc, 0), rc);
  if (nb > 0 && !src) return set_err(GOFFT_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(p->mu);
  if (int e = ensure_staging(p, (size_t)rc * 16, (size_t)p->total * 8)) return e;
  if (nb > 0) GF_CK(cudaMemcpyAsync(p->d_in, src, (size_t)nb * 16, cudaMemcpyHostToDevice, p->stream));
  if (int e = p->rx->c2r(contig(p->d_in, rc), (int)nb, contig(p->d_out, p->total), 1, 1.0, p->ws, p->stream)) return e;
  GF_CK(cudaMemcpyAsync(dst, p->d_out, (size_t)p->total * 8, cudaMemcpyDeviceToHost, p->stream));
  GF_CK(cudaStreamSynchronize(p->stream));
  return GOFFT_OK;
}

extern "C" int gofft_fft(const double *x, int64_t n, double *out) {
  if (n < 0) return set_err(GOFFT_EINVAL, "fft: negative length");
  if (n <= 1) {
    if (n == 1) memmove(out, x, 16);
    return GOFFT_OK;
  }
  gofft_plan *p = nullptr;
  if (int e = gofft_cached_plan(n, &p)) return e;
  return gofft_plan_fft(p, out, x);
}
extern "C" int gofft_ifft(const double *x, int64_t n, double *out) {
  if (n < 0) return set_err(GOFFT_EINVAL, "fft: negative length");
  if (n <= 1) {
    if (n == 1) memmove(out, x, 16);
    return GOFFT_OK;
  }
  gofft_plan *p = nullptr;
  if (int e = gofft_cached_plan(n, &p)) return e;
  return gofft_plan_ifft(p, out, x);
}
extern "C" int gofft_fft_real(const double *x, int64_t n, double *out) {
  if (n < 0) return set_err(GOFFT_EINVAL, "fft: negative length");
  std::vector<double> c((size_t)2 * n, 0.0);
  for (int64_t i = 0; i < n; i++) c[2 * i] = x[i];
  return gofft_fft(c.data(), n, out);
}

extern "C" int gofft_rfft(const double *x, int64_t n, double *out) {
  if (n < 0) return set_err(GOFFT_EINVAL, "fft: negative length");
  if (n == 0) return GOFFT_OK;
  gofft_plan *p = memo(g_rplans, g_rmu, n, true);
  if (!p) return GOFFT_ECUDA;
  return gofft_real_plan_rfft(p, out, x);
}
extern "C" int gofft_irfft(const double *spectrum, int64_t nspec, int64_t n, double *out) {
  if (n <= 0) return GOFFT_OK;
  gofft_plan *p = memo(g_rplans, g_rmu, n, true);
  if (!p) return GOFFT_ECUDA;
  return gofft_real_plan_irfft(p, out, spectrum, nspec);
}

// N-D plans memoised by (kind, shape).
static std::mutex g_nmu;
static std::map<std::pair<int, std::vector<long long>>, gofft_plan *> g_nplans;
static gofft_plan *nd_plan(int kind, const std::vector<long long> &shape) {
  auto key = std::make_pair(kind, shape);
  {
    std::lock_guard<std::mutex> lk(g_nmu);
    auto it = g_nplans.find(key);
    if (it != g_nplans.end()) return it->second;
  }
  gofft_plan *p = nullptr;
  std::vector<int64_t> sh(shape.begin(), shape.end());
  if (gofft_plan_create(kind, GOFFT_F64, sh.data(), (int)sh.size(), 1, 1, 0, 1, 0, &p) != GOFFT_OK) return nullptr;
  p->cached = true;
  std::lock_guard<std::mutex> lk(g_nmu);
  auto it = g_nplans.find(key);
  if (it != g_nplans.end()) {
    p->cached = false;
    delete p;
    return it->second;
  }
  g_nplans[key] = p;
  return p;
}

// ndfft.go:50-62
static int validate_shape(const int64_t *shape, int rank, int64_t len) {
  long long prod = 1;
  for (int a = 0; a < rank; a++) {
    if (shape[a] <= 0) return set_err(GOFFT_EINVAL, "fft: shape lengths must be positive");
    prod *= shape[a];
  }
  if (prod != len) return set_err(GOFFT_EINVAL, "fft: shape product does not match len(data)");
  return GOFFT_OK;
}

static int fftn_impl(const double *data, int64_t len, const int64_t *shape, int rank, double *out, int inverse) {
  if (rank < 0 || (rank > 0 && !shape)) return set_err(GOFFT_EINVAL, "bad rank");
  if (int e = validate_shape(shape, rank, len)) return e;
  if (len <= 1) {
    if (len == 1) memmove(out, data, 16);
    return GOFFT_OK;
  }
  gofft_plan *p = nd_plan(GOFFT_C2C, std::vector<long long>(shape, shape + rank));
  if (!p) return GOFFT_ECUDA;
  return gofft_exec_c2c_host(p, data, out, inverse);
}
extern "C" int gofft_fftn(const double *data, int64_t len, const int64_t *shape, int rank, double *out) {
  return fftn_impl(data, len, shape, rank, out, 0);
}
extern "C" int gofft_ifftn(const double *data, int64_t len, const int64_t *shape, int rank, double *out) {
  return fftn_impl(data, len, shape, rank, out, 1);
}
extern "C" int gofft_fft2(const double *data, int64_t len, int64_t rows, int64_t cols, double *out) {
  const int64_t sh[2] = {rows, cols};
  return fftn_impl(data, len, sh, 2, out, 0);
}
extern "C" int gofft_ifft2(const double *data, int64_t len, int64_t rows, int64_t cols, double *out) {
  const int64_t sh[2] = {rows, cols};
  return fftn_impl(data, len, sh, 2, out, 1);
}

extern "C" int gofft_rfft2(const double *data, int64_t len, int64_t rows, int64_t cols, double *out) {
  if (rows <= 0 || cols <= 0) return set_err(GOFFT_EINVAL, "fft: shape lengths must be positive");
  if (rows * cols != len) return set_err(GOFFT_EINVAL, "fft: shape product does not match len(data)");
  gofft_plan *p = nd_plan(GOFFT_R2C, {rows, cols});
  if (!p) return GOFFT_ECUDA;
  return gofft_exec_r2c_host(p, data, out);
}

extern "C" int gofft_irfft2(const double *data, int64_t len, int64_t rows, int64_t cols, double *out) {
  if (rows <= 0 || cols <= 0) return set_err(GOFFT_EINVAL, "fft: shape lengths must be positive");
  const long long need = rows * (cols / 2 + 1);
  gofft_plan *p = nd_plan(GOFFT_R2C, {rows, cols});
  if (!p) return GOFFT_ECUDA;
  if (len >= need) return gofft_exec_c2r_host(p, data, 0, out);
  // short spectrum: missing bins are zero (rfft2.go:94-99)
  std::vector<double> pad((size_t)need * 2, 0.0);
  if (len > 0) memcpy(pad.data(), data, (size_t)len * 16);
  return gofft_exec_c2r_host(p, pad.data(), 0, out);
}

// window.go:20-22, 59-78
extern "C" int gofft_hann(int64_t n, double *out) {
  if (n <= 0) return GOFFT_OK;
  if (n == 1) {
    out[0] = 1;
    return GOFFT_OK;
  }
  const double denom = (double)(n - 1);
  for (int64_t k = 0; k < n; k++) out[k] = 0.5 + (-1.0) * 0.5 * cos(2 * M_PI * 1.0 * (double)k / denom);
  return GOFFT_OK;
}

// The other symmetric windows (window.go:29-100), on the host in FP64 exactly
// as the reference writes them.
static int cosine_window_host(int64_t n, const double *a, int na, double *out) {
  if (n <= 0) return GOFFT_OK;
  if (!out) return set_err(GOFFT_EINVAL, "null output");
  if (n == 1) {
    out[0] = 1;
    return GOFFT_OK;
  }
  const double denom = (double)(n - 1);
  for (int64_t k = 0; k < n; k++) {
    double s = a[0], sign = -1.0;
    for (int j = 1; j < na; j++) {
      s += sign * a[j] * cos(2 * M_PI * (double)j * (double)k / denom);
      sign = -sign;
    }
    out[k] = s;
  }
  return GOFFT_OK;
}
extern "C" int gofft_hamming(int64_t n, double *out) {
  const double a[2] = {0.54, 0.46};
  return cosine_window_host(n, a, 2, out);
}
extern "C" int gofft_blackman(int64_t n, double *out) {
  const double a[3] = {0.42, 0.5, 0.08};
  return cosine_window_host(n, a, 3, out);
}
extern "C" int gofft_blackman_harris(int64_t n, double *out) {
  const double a[4] = {0.35875, 0.48829, 0.14128, 0.01168};
  return cosine_window_host(n, a, 4, out);
}
extern "C" int gofft_bartlett(int64_t n, double *out) {
  if (n <= 0) return GOFFT_OK;
  if (!out) return set_err(GOFFT_EINVAL, "null output");
  if (n == 1) {
    out[0] = 1;
    return GOFFT_OK;
  }
  const double denom = (double)(n - 1), half = denom / 2;
  for (int64_t k = 0; k < n; k++) out[k] = (2 / denom) * (half - fabs((double)k - half));
  return GOFFT_OK;
}

// FFTFreq / RFFTFreq (freq.go:17-56).
extern "C" int gofft_fftfreq(int64_t n, double d, double *out) {
  if (n <= 0) return GOFFT_OK;
  if (!out) return set_err(GOFFT_EINVAL, "null output");
  const double val = 1.0 / (d * (double)n);
  const int64_t half = (n - 1) / 2;
  for (int64_t i = 0; i <= half; i++) out[i] = (double)i * val;
  int64_t j = -(n / 2);
  for (int64_t i = half + 1; i < n; i++, j++) out[i] = (double)j * val;
  return GOFFT_OK;
}
extern "C" int gofft_rfftfreq(int64_t n, double d, double *out) {
  if (n <= 0) return GOFFT_OK;
  if (!out) return set_err(GOFFT_EINVAL, "null output");
  const double val = 1.0 / (d * (double)n);
  for (int64_t i = 0; i < n / 2 + 1; i++) out[i] = (double)i * val;
  return GOFFT_OK;
}

// Device windows, generated once per (device, precision, kind, length) and
// kept for the process: the spectrogram's fused first stage reads them.
static const void *device_window(int prec, int kind, int64_t n, cudaStream_t st) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int64_t>, void *> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_tuple(dev, prec, kind, n);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  void *w = nullptr;
  const int rb = prec == F64 ? 8 : 4;
  if (cudaMalloc(&w, (size_t)n * rb) != cudaSuccess) {
    set_err(GOFFT_ENOMEM, "window buffer");
    return nullptr;
  }
  if (gen_window(w, rb, n, kind, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
    cudaFree(w);
    set_err(GOFFT_ECUDA, "window generation failed");
    return nullptr;
  }
  cache[key] = w;
  return w;
}

extern "C" int gofft_window_device(int precision, int kind, int64_t n, void *out, gofft_stream stream) {
  if (precision < 0 || precision > 2 || kind < 0 || kind > 4) return set_err(GOFFT_EINVAL, "bad window arguments");
  if (n <= 0) return GOFFT_OK;
  if (!out) return set_err(GOFFT_EINVAL, "null output");
  GF_CK(gen_window(out, precision == F64 ? 8 : 4, n, kind, (cudaStream_t)stream));
  return GOFFT_OK;
}

// Spectrogram frames on device buffers (freq.go:107-127 for even segments).
static int spectro_dev(int prec, const void *x, int64_t nx, int64_t seg, int64_t overlap, const void *win,
                       double d, void *out, int64_t frames, cudaStream_t st) {
  if (frames <= 0) return GOFFT_OK;
  const long long m = seg / 2;
  auto rx = get_real(seg, prec);
  if (!rx) return GOFFT_ECUDA;
  if (rx->mode != R_PACKED_FUSED) return set_err(GOFFT_EUNSUPPORTED, "segment too long for the fused spectrogram");
  KArgs a{};
  a.in = mk_side((void *)x, seg - overlap, 0, 1, 1);
  a.out = mk_side(out, m + 1, 0, 1, 1);
  a.aux0 = rx->tw2;
  a.aux2 = rx->tw2_hi;
  a.aux1 = win;
  a.scale = d / (double)seg;
  a.ic = pairs_aligned(a.in, prec) ? GF_PAIR_ALIGNED : 0;
  (void)nx;
  return launch_line(OP_SPECTRO, *rx->cx->prog, a, frames, st);
}

static int64_t frame_count(int64_t nx, int64_t seg, int64_t overlap) {
  const int64_t step = seg - overlap;
  if (nx < seg) return 0;
  return (nx - seg) / step + 1;
}

extern "C" int gofft_spectrogram_device(int precision, const void *x, int64_t nx, int64_t segment,
                                        int64_t overlap, const void *window, double d, void *out,
                                        int64_t *nframes, gofft_stream stream) {
  if (segment <= 0) return set_err(GOFFT_EINVAL, "fft: segment length must be positive");
  if (overlap < 0 || overlap >= segment) return set_err(GOFFT_EINVAL, "fft: overlap must satisfy 0 <= overlap < segment");
  if (segment % 2) return set_err(GOFFT_EUNSUPPORTED, "device spectrogram needs an even segment");
  if (precision < 0 || precision > 2) return set_err(GOFFT_EINVAL, "bad precision");
  const int64_t frames = frame_count(nx, segment, overlap);
  if (nframes) *nframes = frames;
  if (!out) return GOFFT_OK;
  return spectro_dev(precision, x, nx, segment, overlap, window, d, out, frames, (cudaStream_t)stream);
}

extern "C" int gofft_spectrogram_window_device(int precision, const void *x, int64_t nx, int64_t segment,
                                               int64_t overlap, int window_kind, double d, void *out,
                                               int64_t *nframes, gofft_stream stream) {
  if (window_kind < 0 || window_kind > 4) return set_err(GOFFT_EINVAL, "bad window kind");
  if (segment <= 0) return set_err(GOFFT_EINVAL, "fft: segment length must be positive");
  const void *w = device_window(precision, window_kind, segment, (cudaStream_t)stream);
  if (!w) return GOFFT_ECUDA;
  return gofft_spectrogram_device(precision, x, nx, segment, overlap, w, d, out, nframes, stream);
}

// PSD (freq.go:69-90) of one host signal.
extern "C" int gofft_psd(const double *x, int64_t n, double d, double *out) {
  if (n <= 0) return GOFFT_OK;
  const int64_t m = n / 2 + 1;
  std::vector<double> spec((size_t)2 * m);
  if (int e = gofft_rfft(x, n, spec.data())) return e;
  const double scale = d / (double)n;
  for (int64_t k = 0; k < m; k++) {
    const double re = spec[2 * k], im = spec[2 * k + 1];
    double pw = (re * re + im * im) * scale;
    if (k != 0 && !(n % 2 == 0 && k == m - 1)) pw *= 2;
    out[k] = pw;
  }
  return GOFFT_OK;
}

extern "C" int gofft_spectrogram(const double *x, int64_t nx, int64_t segment, int64_t overlap,
                                 const double *window, int64_t nwindow, double d, double *out,
                                 int64_t *nframes) {
  if (segment <= 0) return set_err(GOFFT_EINVAL, "fft: segment length must be positive");
  if (nwindow != segment) return set_err(GOFFT_EINVAL, "fft: window length must equal segment length");
  if (overlap < 0 || overlap >= segment) return set_err(GOFFT_EINVAL, "fft: overlap must satisfy 0 <= overlap < segment");
  const int64_t frames = frame_count(nx, segment, overlap);
  if (nframes) *nframes = frames;
  if (!out || frames == 0) return GOFFT_OK;
  const int64_t bins = segment / 2 + 1;
  if (segment % 2 == 0 && get_real(segment, F64) && get_real(segment, F64)->mode == R_PACKED_FUSED) {
    void *dx = nullptr, *dw = nullptr, *dout = nullptr;
    const size_t used = (size_t)((frames - 1) * (segment - overlap) + segment);
    int rc = GOFFT_OK;
    if (cudaMalloc(&dx, used * 8) != cudaSuccess || cudaMalloc(&dw, segment * 8) != cudaSuccess ||
        cudaMalloc(&dout, (size_t)frames * bins * 8) != cudaSuccess) {
      rc = set_err(GOFFT_ENOMEM, "spectrogram buffers");
    } else {
      cudaMemcpy(dx, x, used * 8, cudaMemcpyHostToDevice);
      cudaMemcpy(dw, window, segment * 8, cudaMemcpyHostToDevice);
      rc = spectro_dev(F64, dx, nx, segment, overlap, dw, d, dout, frames, 0);
      if (rc == GOFFT_OK) {
        cudaError_t e = cudaMemcpy(out, dout, (size_t)frames * bins * 8, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = set_err(GOFFT_ECUDA, cudaGetErrorString(e));
      }
    }
    cudaFree(dx);
    cudaFree(dw);
    cudaFree(dout);
    return rc;
  }
  // odd (or over-long) segments: one PSD per windowed frame
  std::vector<double> seg((size_t)segment);
  for (int64_t t = 0; t < frames; t++) {
    const int64_t start = t * (segment - overlap);
    for (int64_t i = 0; i < segment; i++) seg[i] = x[start + i] * window[i];
    if (int e = gofft_psd(seg.data(), segment, d, out + t * bins)) return e;
  }
  return GOFFT_OK;
}

// ---------------------------------------------------------------------------
// Instrumentation
// ---------------------------------------------------------------------------
extern "C" int64_t gofft_launch_count(void) { return launch_count(); }
extern "C" int gofft_timing_enable(int on) {
  timing_enable(on);
  return GOFFT_OK;
}
extern "C" int64_t gofft_timing_report(char *buf, int64_t cap) {
  static thread_local std::string last;
  if (!buf || cap <= 0) {
    last = timing_report();
    return (int64_t)last.size();
  }
  const size_t k = std::min<size_t>(last.size(), (size_t)cap - 1);
  memcpy(buf, last.data(), k);
  buf[k] = 0;
  return (int64_t)last.size();
}
extern "C" int gofft_set_lines_per_cta(int precision, int64_t n, int op, int colmode, int lpc) {
  set_lpc_override(precision, n, op, colmode, lpc);
  return GOFFT_OK;
}
extern "C" int gofft_set_l2_block_bytes(int64_t bytes) {
  g_l2_block_bytes.store(bytes > 0 ? bytes : kL2BlockBytes);
  return GOFFT_OK;
}
extern "C" int gofft_set_lanes(int lanes) {
  if (lanes < 0 || lanes > 2) return set_err(GOFFT_EINVAL, "lanes must be 1 or 2 (0: the default)");
  g_lanes.store(lanes == 0 ? kLanes : lanes);
  return GOFFT_OK;
}
extern "C" int gofft_set_tma_pipeline(int on) {
  set_tma_pipeline(on);
  return GOFFT_OK;
}
extern "C" int gofft_pipeline_status(void) { return pipe_status(true); }
extern "C" int gofft_set_dependent_launch(int mode) {
  if (mode < 0 || mode > 2) return set_err(GOFFT_EINVAL, "dependent-launch mode must be 0, 1 or 2");
  set_dependent_launch(mode);
  return GOFFT_OK;
}
extern "C" int gofft_set_pipelined(int precision, int64_t n, int op, int on) {
  set_pipe_override(precision, n, op, on);
  return GOFFT_OK;
}

extern "C" int gofft_set_schedule(int precision, int64_t n, int variant) {
  if (precision < 0 || precision > 2 || n < 1 || variant < 0 || variant > 2)
    return set_err(GOFFT_EINVAL, "bad schedule override");
  set_sched_variant(precision, n, variant);
  return GOFFT_OK;
}

extern "C" int gofft_get_schedule(int precision, int64_t n) { return get_sched_variant(precision, n); }

// ---------------------------------------------------------------------------
// CUDA graphs
// ---------------------------------------------------------------------------
struct gofft_graph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  ~gofft_graph() {
    if (x) cudaGraphExecDestroy(x);
    if (g) cudaGraphDestroy(g);
  }
};

extern "C" int gofft_graph_begin(gofft_stream stream) {
  if (!stream) return set_err(GOFFT_EINVAL, "capture needs a non-default stream");
  GF_CK(cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal));
  return GOFFT_OK;
}
extern "C" int gofft_graph_end(gofft_stream stream, gofft_graph **out) {
  if (!out) return set_err(GOFFT_EINVAL, "null output handle");
  std::unique_ptr<gofft_graph> g(new gofft_graph());
  GF_CK(cudaStreamEndCapture((cudaStream_t)stream, &g->g));
  GF_CK(cudaGraphInstantiate(&g->x, g->g, 0));
  *out = g.release();
  return GOFFT_OK;
}
extern "C" int gofft_graph_launch(gofft_graph *g, gofft_stream stream) {
  if (!g) return set_err(GOFFT_EINVAL, "null graph");
  GF_CK(cudaGraphLaunch(g->x, (cudaStream_t)stream));
  return GOFFT_OK;
}
extern "C" int gofft_graph_destroy(gofft_graph *g) {
  delete g;
  return GOFFT_OK;
}

// ---------------------------------------------------------------------------
// Adjoints (vector-Jacobian products).  No counterpart in the reference.  The
// inner product is the real one, Re sum conj(a) b, so a complex gradient
// holds dL/dRe + i dL/dIm (torch's convention for real losses).
// ---------------------------------------------------------------------------
extern "C" int gofft_vjp_c2c(gofft_plan *p, const void *g, void *out, int inverse, gofft_stream stream) {
  if (!p || !g || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_C2C) return set_err(GOFFT_EINVAL, "plan is not complex-to-complex");
  // FFT^H = N IFFT = conj(FFT(conj .)) unscaled; IFFT^H = FFT / N.  Both are
  // the opposite direction with the inverse's scaling.
  return exec_c2c_dir(p, g, out, inverse ? 0 : 1, inverse ? 1 : 0, (cudaStream_t)stream);
}

extern "C" int gofft_vjp_r2c(gofft_plan *p, const void *g, void *out, gofft_stream stream) {
  if (!p || !g || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_R2C) return set_err(GOFFT_EINVAL, "plan is not real");
  // RFFT^T(G) = N IRFFT(G / w): the unnormalised inverse with interior bins halved
  return exec_c2r(p, g, 0, out, (cudaStream_t)stream, true);
}

extern "C" int gofft_vjp_c2r(gofft_plan *p, const void *g, void *out, gofft_stream stream) {
  if (!p || !g || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_R2C) return set_err(GOFFT_EINVAL, "plan is not real");
  // IRFFT^T(g) = (w / N) RFFT(g)
  return exec_r2c(p, g, out, (cudaStream_t)stream, 1.0 / (double)p->total);
}

// y = IRFFT2(H * RFFT2(x)) per image, and its adjoint, in three passes per L2
// block of images: rows R2C into the block buffer, one fused column pass
// (column FFT, multiply, column IFFT -- OpFilterCol) in place, rows C2R.
static int filter2_run(gofft_plan *p, const void *x, const void *H, void *y, void *saved, void *part, int fl,
                       cudaStream_t st) {
  const long long rows = p->shape[0], cols = p->shape[1], rc = cols / 2 + 1;
  const size_t r = rsize(p->prec), c = csize(p->prec);
  const long long per = rows * rc;
  const Exec1D &cx = *p->ax[0];
  const double dsc = 1.0 / ((double)rows * (double)cols);
  Lanes ln(p, st);
  if (int e = ln.fork((p->batch + p->chunk - 1) / p->chunk)) return e;
  long long blk = -1;
  for (long long b0 = 0; b0 < p->batch; b0 += p->chunk) {
    blk++;
    const long long nb = std::min(p->chunk, p->batch - b0);
    const cudaStream_t s = ln.stream(blk);
    char *spec = ln.buf(blk);
    char *wsx = ln.sub(blk);
    const char *src = (const char *)x + (size_t)b0 * rows * cols * r;
    char *sv = saved ? (char *)saved + (size_t)b0 * per * c : nullptr;
    char *pt = part ? (char *)part + (size_t)b0 * per * c : nullptr;
    if (int e = p->rx->r2c(contig((void *)src, cols), contig(spec, rc), nb * rows, wsx, s)) return ln.join(e);
    const Side cs = mk_side(spec, per, 1, rc, rc);
    if (rows > 1 && cx.kind == K_SINGLE) {
      KArgs a{};
      a.in = cs;
      a.out = cs;
      a.aux0 = H;
      a.aux1 = sv;
      a.aux2 = pt;
      a.ia = cols;
      a.ic = fl;
      a.da = dsc;
      a.cj_out = 1;
      a.scale = 1.0 / (double)rows;
      if (int e = launch_line(OP_FILTER_COL, *cx.prog, a, nb * rc, s, 0, true)) return ln.join(e);
    } else {
      if (rows > 1)
        if (int e = cx.exec(cs, cs, nb * rc, 0, 0, 1.0, wsx, s)) return ln.join(e);
      if (GF_PREC_CALL(p->prec, filter_ew, spec, H, sv, pt, nb, rows, rc, cols, fl, dsc, s) != cudaSuccess)
        return ln.join(set_err(GOFFT_ECUDA, "filter kernel launch failed"));
      if (rows > 1)
        if (int e = cx.exec(cs, cs, nb * rc, 1, 1, 1.0 / (double)rows, wsx, s)) return ln.join(e);
    }
    if (y) {
      char *dst = (char *)y + (size_t)b0 * rows * cols * r;
      if (int e = p->rx->c2r(contig(spec, rc), (int)rc, contig(dst, cols), nb * rows, 1.0, wsx, s)) return ln.join(e);
    }
  }
  return ln.join(GOFFT_OK);
}

static int filter2_check(gofft_plan *p) {
  if (!p) return set_err(GOFFT_EINVAL, "null plan");
  if (p->kind != GOFFT_R2C || p->rank != 2)
    return set_err(GOFFT_EINVAL, "the 2-D spectral filter needs a rank-2 real plan");
  return GOFFT_OK;
}

extern "C" int gofft_filter2_forward(gofft_plan *p, const void *x, const void *H, void *y, void *saved,
                                     gofft_stream stream) {
  if (int e = filter2_check(p)) return e;
  if (!x || !H || !y) return set_err(GOFFT_EINVAL, "null argument");
  return filter2_run(p, x, H, y, saved, nullptr, saved ? GF_FILT_SAVE : 0, (cudaStream_t)stream);
}

extern "C" int gofft_vjp_filter2(gofft_plan *p, const void *g, const void *H, const void *saved, void *scratch,
                                 void *dx, void *dH, gofft_stream stream) {
  if (int e = filter2_check(p)) return e;
  if (!g || !H) return set_err(GOFFT_EINVAL, "null argument");
  if (!dx && !dH) return GOFFT_OK;
  if (dH && (!saved || !scratch))
    return set_err(GOFFT_EINVAL, "dH needs the forward's saved spectra and a scratch buffer");
  const cudaStream_t st = (cudaStream_t)stream;
  // dx = IRFFT2(conj(H) * RFFT2(g)); dH = sum_b conj(X_b) * (w / (R C)) * RFFT2(g_b)
  if (dH && saved != scratch) {
    const size_t bytes = (size_t)p->batch * p->shape[0] * (p->shape[1] / 2 + 1) * csize(p->prec);
    GF_CK(cudaMemcpyAsync(scratch, saved, bytes, cudaMemcpyDeviceToDevice, st));
  }
  const int fl = GF_FILT_CONJ | (dH ? GF_FILT_DH : 0);
  if (int e = filter2_run(p, g, H, dx, dH ? scratch : nullptr, dH ? scratch : nullptr, fl, st)) return e;
  if (dH) {
    const long long count = p->shape[0] * (p->shape[1] / 2 + 1);
    GF_CK(GF_PREC_CALL(p->prec, sum_batches, dH, scratch, count, p->batch, st));
  }
  return GOFFT_OK;
}

// ---------------------------------------------------------------------------
// Complex transform that allocates nothing.
//
// gofft_exec_c2c() runs multi-pass transforms (lengths split into two passes,
// and primes whose convolution is split) through the plan's own workspace.
// Some callers cannot have any device memory allocated on their behalf while
// they run: code that records work into a CUDA graph (allocation calls are not
// part of the captured stream and can invalidate the capture), programs whose
// device memory is owned and budgeted by another allocator's pool, and paths
// where the device-wide synchronisation of cudaMalloc/cudaFree is not
// acceptable.  For them this entry point takes its scratch from one
// fixed-size array that is part of the library image: it never calls
// cudaMalloc, cudaFree or any allocating routine.
//
// The array, kNoAllocScratchBytes (16 MiB), is held by every GPU that loads
// the library until the process exits.  Host code cannot use the symbol's
// address directly (it names a host-side stand-in), so the device address is
// looked up once per device with cudaGetSymbolAddress, by the first call on
// that device; make that first call before starting any stream capture.
// Every call uses the same array and it keeps whatever the last call left:
// nothing in it needs to start at zero (each pass writes all the scratch it
// later reads), but calls whose executions overlap on the GPU (different
// streams, or different threads) race on it and must be serialised by the
// caller.
// ---------------------------------------------------------------------------
static constexpr size_t kNoAllocScratchBytes = 16u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static std::map<int, void *> g_noalloc_addr;

extern "C" int gofft_exec_c2c_noalloc(gofft_plan *p, const void *in, void *out, int inverse,
                                      gofft_stream stream) {
  if (!p || !in || !out) return set_err(GOFFT_EINVAL, "null argument");
  if (p->kind != GOFFT_C2C) return set_err(GOFFT_EINVAL, "plan is not complex-to-complex");
  if (p->rank != 1) return set_err(GOFFT_EUNSUPPORTED, "the no-allocation entry point takes 1-D complex plans");
  const size_t need = p->ax[0]->ws_bytes(p->batch);
  if (need > kNoAllocScratchBytes)
    return set_err(GOFFT_EINVAL, "transform needs " + std::to_string(need) +
                                     " bytes of scratch; the no-allocation entry point has " +
                                     std::to_string(kNoAllocScratchBytes));
  int dev = 0;
  GF_CK(cudaGetDevice(&dev));
  void *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    auto it = g_noalloc_addr.find(dev);
    if (it == g_noalloc_addr.end()) {
      void *ptr = nullptr;
      GF_CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
      it = g_noalloc_addr.emplace(dev, ptr).first;
    }
    scratch = it->second;
  }
  const int cj = inverse ? 1 : 0;
  const double sc = inverse ? 1.0 / (double)p->shape[0] : 1.0;
  return p->ax[0]->exec(mk_side((void *)in, p->idist, 0, p->istride, 1), mk_side(out, p->odist, 0, p->ostride, 1),
                        p->batch, cj, cj, sc, need ? scratch : nullptr, (cudaStream_t)stream);
}
