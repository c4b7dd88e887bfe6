// ppf_api.cu -- the extern "C" entry points of libppf.so (declared in
// include/ppf.h): argument validation, workspace layout and path choice.
#include <cuda_runtime.h>

#include <algorithm>
#include <math.h>
#include <string.h>

#include "ppf.h"
#include "ppf_core.cuh"
#include "ppf_detmath.h"
#include "ppf_internal.h"

namespace ppf {

static size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// Carve the workspace for `path`; with base == nullptr only sizes are computed.
static size_t carve(Args& a, int path, unsigned char* base) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> unsigned char* {
    unsigned char* p = base ? base + off : nullptr;
    off = align_up(off + bytes);
    return p;
  };
  const int dx = a.model.dx;
  a.err = reinterpret_cast<uint32_t*>(take(64));
  a.counter = reinterpret_cast<unsigned int*>(base ? base + 16 : nullptr);
  a.gbar = reinterpret_cast<unsigned int*>(base ? base + 32 : nullptr);
  if (path == PPF_PATH_STREAM) {
    // a.tile is chosen before carving; the per-tile arrays are sized for the
    // smallest tile so that one workspace serves every tile configuration
    if (a.tile != kTileLarge && a.tile != kTileMid && a.tile != kTileSmall) a.tile = kTileLarge;
    a.ntiles = (a.J + a.tile - 1) / a.tile;
    const size_t nt_alloc = (size_t)(a.J + kTileSmall - 1) / kTileSmall;
    for (int i = 0; i < 2; ++i) a.acc[i] = reinterpret_cast<Acc*>(take(sizeof(Acc) * a.F));
    for (int i = 0; i < 2; ++i) a.desc[i] = reinterpret_cast<uint64_t*>(take(8ull * a.F * nt_alloc));
    a.excl = reinterpret_cast<uint64_t*>(take(8ull * a.F * nt_alloc));
    a.tot = reinterpret_cast<uint64_t*>(take(8ull * a.F));
    for (int i = 0; i < 2; ++i) a.fdone[i] = reinterpret_cast<unsigned int*>(take(4ull * a.F));
    a.ctrl_bytes = off;
    a.consts = take((lg_wide(a.model) ? 2048ull : 512ull) * a.F);
    // per-thread run prefixes: ntiles x threads per tile, the largest over the tile configurations
    const size_t J = (size_t)a.J;
    const size_t nrun = std::max({(J + kTileLarge - 1) / kTileLarge * 256, (J + kTileMid - 1) / kTileMid * 128,
                                  (J + kTileSmall - 1) / kTileSmall * 64});
    a.runpre = reinterpret_cast<uint64_t*>(take(8ull * a.F * nrun));
    for (int i = 0; i < 2; ++i) a.X[i] = reinterpret_cast<float*>(take(4ull * a.F * dx * a.J));
    for (int i = 0; i < 2; ++i) a.W[i] = reinterpret_cast<float*>(take(4ull * a.F * a.J));
  } else if (path == PPF_PATH_PLAIN) {
    const int nblk = (a.J + 255) / 256;
    for (int i = 0; i < 2; ++i) a.acc[i] = reinterpret_cast<Acc*>(take(sizeof(Acc)));
    a.tot = reinterpret_cast<uint64_t*>(take(8));
    a.pl_carry_dev = reinterpret_cast<int*>(take(4));
    a.ctrl_bytes = off;
    for (int i = 0; i < 2; ++i) a.X[i] = reinterpret_cast<float*>(take(4ull * dx * a.J));
    for (int i = 0; i < 2; ++i) a.W[i] = reinterpret_cast<float*>(take(4ull * a.J));
    a.pl_cdf = reinterpret_cast<uint64_t*>(take(8ull * a.J));
    a.pl_bsum = reinterpret_cast<uint64_t*>(take(8ull * nblk));
    a.pl_boff = reinterpret_cast<uint64_t*>(take(8ull * nblk));
    a.pl_anc = reinterpret_cast<int*>(take(4ull * a.J));
  } else {
    a.ctrl_bytes = off;
  }
  return off;
}

static int n_params_of(const ppf_model& m) {
  switch (m.kind) {
    case PPF_MODEL_LG:
      return m.dx * m.dx + m.dy * m.dx + m.dx * (m.dx + 1) / 2 + m.dy * (m.dy + 1) / 2 + m.dx;
    case PPF_MODEL_SV: return 6;
    case PPF_MODEL_RICKER: return 4;
    default: return -1;
  }
}

static int check_model(const ppf_model& m) {
  switch (m.kind) {
    case PPF_MODEL_LG:
      if (m.dx < 1 || m.dx > 9 || m.dy < 1 || m.dy > 9) return PPF_EINVAL;   // linear_gaussian.py:48 MAX_DIM
      break;
    case PPF_MODEL_SV:
      if (m.dx != 2 || m.dy != 1 || !(m.dt > 0.0f)) return PPF_EINVAL;
      break;
    case PPF_MODEL_RICKER:
      if (m.dx != 1 || m.dy != 1) return PPF_EINVAL;
      break;
    default: return PPF_EINVAL;
  }
  if (m.n_params != n_params_of(m)) return PPF_EINVAL;
  return PPF_OK;
}

static int choose_path(const ppf_pfilter_desc* d) {
  if (d->path != PPF_PATH_AUTO) return d->path;
  Args a{};
  a.J = d->J; a.F = d->F; a.flags = d->flags; a.model = d->model; a.mode = MODE_PF;
  // the wide LG streams only
  if (lg_wide(d->model)) return PPF_PATH_STREAM;
  // swarm fits one CTA's shared memory: keep it on chip for the whole loop.
  // Up to J = 8192: at J = 16384 (1024 Ricker filters) the streaming kernels
  // take 179 ms against the resident kernel's 259 ms (one 512-thread CTA per
  // SM holds such a swarm, too few warps to hide its latencies)
  const bool resident = resident_smem_bytes(a) <= kResidentSmemMax && d->J <= 8192;
  if (resident && d->F >= kNumSMs) return PPF_PATH_RESIDENT;
  // few filters of a few thousand particles or more: the streaming kernels
  // would leave most SMs idle; a cluster per filter keeps the swarm on chip
  // (when all filters' clusters are resident at once)
  const long long tiles = (long long)d->F * ((d->J + kTileLarge - 1) / kTileLarge);
  if (d->J > 2048 && tiles < 2LL * kNumSMs && cluster_fits(a, false)) return PPF_PATH_CLUSTER;
  if (resident) return PPF_PATH_RESIDENT;
  return PPF_PATH_STREAM;
}

// ---------------------------------------------------------------------------
// Tile choice: an explicit desc->tile, else a measured choice from
// ppf_autotune for the same shape, else the smallest tile that still gives
// two CTAs per SM (more, smaller CTAs when there are few particles).
// ---------------------------------------------------------------------------
struct TuneEntry {
  int kind, dx, dy, J, F, U, inj, tile;
};
constexpr int kTuneCap = 64;
static TuneEntry g_tune[kTuneCap];
static int g_tune_n = 0;

static int tune_lookup(const ppf_model& m, int J, int F, int U, int inj) {
  for (int i = 0; i < g_tune_n; ++i) {
    const TuneEntry& e = g_tune[i];
    if (e.kind == m.kind && e.dx == m.dx && e.dy == m.dy && e.J == J && e.F == F && e.U == U && e.inj == inj)
      return e.tile;
  }
  return 0;
}

static void tune_store(const ppf_model& m, int J, int F, int U, int inj, int tile) {
  for (int i = 0; i < g_tune_n; ++i) {
    TuneEntry& e = g_tune[i];
    if (e.kind == m.kind && e.dx == m.dx && e.dy == m.dy && e.J == J && e.F == F && e.U == U && e.inj == inj) {
      e.tile = tile;
      return;
    }
  }
  TuneEntry e{m.kind, m.dx, m.dy, J, F, U, inj, tile};
  g_tune[g_tune_n < kTuneCap ? g_tune_n++ : (kTuneCap - 1)] = e;
}

static int choose_tile(const ppf_model& m, int J, int F, int U, int inj, int requested) {
  if (lg_wide(m)) return kTileSmall;   // the wide LG has one tile configuration
  if (requested == kTileLarge || requested == kTileMid || requested == kTileSmall) return requested;
  const int tuned = tune_lookup(m, J, F, U, inj);
  if (tuned) return tuned;
  const long long want = 2LL * kNumSMs;
  const int cand[2] = {kTileLarge, kTileMid};
  for (int c : cand)
    if ((long long)F * ((J + c - 1) / c) >= want) return c;
  return kTileSmall;
}

// Polls before a bounded device-side wait gives up (ppf_debug_set_wait_limit).
static long long g_spin_cap = kSpinCap;

static int fill_args(const ppf_pfilter_desc* d, Args& a, int mode) {
  memset(&a, 0, sizeof(a));
  a.pwi = -1;
  a.spin_cap = g_spin_cap;
  a.model = d->model;
  a.J = d->J; a.F = d->F; a.T = d->T; a.U = d->U;
  a.flags = d->flags;
  a.mode = mode;
  a.thresh = d->thresh > 0.0f ? d->thresh : 0.0f;
  a.logthresh = a.thresh > 0.0f ? pp_logf(a.thresh) : -INFINITY;
  a.base_init = pp_logf(1.0f / (float)d->J);
  a.base_rs = -pp_logf((float)d->J);
  a.theta = d->theta; a.ys = d->ys; a.ycon = d->ycon; a.unit = d->unit; a.T_u = d->T_u;
  a.seeds = d->seeds; a.inj_z0 = d->inj_z0; a.inj_z = d->inj_z; a.inj_u = d->inj_u;
  a.loglik = d->loglik;
  a.cll = (d->flags & PPF_F_CLL) ? d->cll : nullptr;
  a.ess = (d->flags & PPF_F_ESS) ? d->ess : nullptr;
  a.fmean = (d->flags & PPF_F_FMEAN) ? d->fmean : nullptr;
  a.pmean = (d->flags & PPF_F_PMEAN) ? d->pmean : nullptr;
  a.anc = (d->flags & PPF_F_SAVE_ANC) ? d->anc : nullptr;
  a.logw = (d->flags & PPF_F_SAVE_W) ? d->logw : nullptr;
  a.tile = choose_tile(d->model, d->J, d->F, d->U, (d->flags & PPF_F_INJECT) ? 1 : 0, d->tile);
  return PPF_OK;
}

static int validate(const ppf_pfilter_desc* d) {
  if (!d) return PPF_EINVAL;
  if (d->J < 1 || d->J > PPF_MAX_J || d->F < 1 || d->T < 1 || d->U < 1) return PPF_EINVAL;
  int rc = check_model(d->model);
  if (rc) return rc;
  if (!d->theta || !d->ys || !d->loglik) return PPF_EINVAL;
  if (!(d->flags & PPF_F_INJECT) && !d->seeds) return PPF_EINVAL;
  if ((d->flags & PPF_F_INJECT) && (!d->inj_z || !d->inj_u)) return PPF_EINVAL;
  if ((d->flags & PPF_F_INJECT) && d->model.kind == PPF_MODEL_LG && !d->inj_z0) return PPF_EINVAL;
  if (d->model.kind == PPF_MODEL_RICKER && !d->ycon) return PPF_EINVAL;
  if ((d->flags & PPF_F_CLL) && !d->cll) return PPF_EINVAL;
  if ((d->flags & PPF_F_ESS) && !d->ess) return PPF_EINVAL;
  if ((d->flags & PPF_F_FMEAN) && !d->fmean) return PPF_EINVAL;
  if ((d->flags & PPF_F_PMEAN) && !d->pmean) return PPF_EINVAL;
  if ((d->flags & PPF_F_SAVE_ANC) && !d->anc) return PPF_EINVAL;
  if ((d->flags & PPF_F_SAVE_W) && !d->logw) return PPF_EINVAL;
  if (d->path < PPF_PATH_AUTO || d->path > PPF_PATH_CLUSTER) return PPF_EINVAL;
  if (d->tile != 0 && d->tile != kTileLarge && d->tile != kTileMid && d->tile != kTileSmall) return PPF_EINVAL;
  return PPF_OK;
}

// MOP: stream-path carve plus the adjoint working set.
static size_t carve_mop(Args& a, MopWork& w, const ppf_mop_desc* d, unsigned char* base) {
  size_t off = carve(a, PPF_PATH_STREAM, base);
  auto take = [&](size_t bytes) -> unsigned char* {
    unsigned char* p = base ? base + off : nullptr;
    off = align_up(off + bytes);
    return p;
  };
  const int dx = a.model.dx;
  const size_t F = a.F, T = a.T, J = a.J;
  int L = d->ckpt_every;
  if (L <= 0) {
    L = 1;
    while ((size_t)L * L < T) ++L;
  }
  a.ckpt_every = L;
  a.nseg = (int)((T + L - 1) / L);
  int32_t* anc = reinterpret_cast<int32_t*>(take(d->anc ? 0 : 4 * F * T * J));
  a.anc = d->anc ? d->anc : anc;
  a.mop_off = reinterpret_cast<int*>(take(4 * F * T * (J + 1)));
  a.mop_ckpt = reinterpret_cast<float*>(take(4 * F * a.nseg * dx * J));
  a.mop_M = reinterpret_cast<float*>(take(4 * F * T));
  a.mop_S = reinterpret_cast<double*>(take(8 * F * T));
  w.sb = reinterpret_cast<float*>(take(4 * F * L * dx * J));
  w.sb2 = reinterpret_cast<float*>(take(4 * F * L * dx * J));
  w.gpart = reinterpret_cast<double*>(take(8 * kMaxNG * F * ((J + 255) / 256)));
  w.lx = reinterpret_cast<float*>(take(4 * 2 * F * dx * J));
  w.lw = reinterpret_cast<float*>(take(4 * 2 * F * J));
  w.gnat = reinterpret_cast<double*>(take(8 * F * kMaxNG));
  a.slotw = reinterpret_cast<uint64_t*>(take(8ull * 6 * kInboxWords));
  return off;
}

static int validate_mop(const ppf_mop_desc* d) {
  if (!d) return PPF_EINVAL;
  if (d->J < 1 || d->J > PPF_MAX_J || d->F < 1 || d->T < 1 || d->U < 1) return PPF_EINVAL;
  int rc = check_model(d->model);
  if (rc) return rc;
  if (!d->theta || !d->ys || !d->value) return PPF_EINVAL;
  if (!(d->flags & PPF_F_INJECT) && !d->seeds) return PPF_EINVAL;
  if ((d->flags & PPF_F_INJECT) && (!d->inj_z || !d->inj_u)) return PPF_EINVAL;
  if ((d->flags & PPF_F_INJECT) && d->model.kind == PPF_MODEL_LG && !d->inj_z0) return PPF_EINVAL;
  if (d->model.kind == PPF_MODEL_RICKER && !d->ycon) return PPF_EINVAL;
  if (!(d->alpha >= 0.0f && d->alpha <= 1.0f)) return PPF_EINVAL;
  if ((d->flags & PPF_F_DPOP) && (d->process_weight_index < 0 || d->process_weight_index >= d->model.dx))
    return PPF_EINVAL;
  return PPF_OK;
}

static void mop_to_pfilter(const ppf_mop_desc* d, ppf_pfilter_desc* p) {
  memset(p, 0, sizeof(*p));
  p->model = d->model;
  p->J = d->J; p->F = d->F; p->T = d->T; p->U = d->U;
  p->path = PPF_PATH_STREAM;
  p->flags = (d->flags & (PPF_F_INJECT | PPF_F_NO_PERSIST)) | ((d->flags & PPF_F_NATURAL) ? 0u : PPF_F_EST);
  p->thresh = 0.0f;
  p->theta = d->theta; p->ys = d->ys; p->ycon = d->ycon; p->unit = d->unit; p->T_u = d->T_u;
  p->seeds = d->seeds; p->inj_z0 = d->inj_z0; p->inj_z = d->inj_z; p->inj_u = d->inj_u;
  p->loglik = d->value;
}

// IF2: stream-path carve plus the two parameter-swarm buffers.
static size_t carve_if2(Args& a, unsigned char* base) {
  size_t off = carve(a, PPF_PATH_STREAM, base);
  for (int i = 0; i < 2; ++i) {
    a.TH[i] = reinterpret_cast<float*>(base ? base + off : nullptr);
    off = align_up(off + 4ull * a.F * a.model.n_params * a.J);
  }
  return off;
}

static int validate_if2(const ppf_perfilter_desc* d) {
  if (!d) return PPF_EINVAL;
  if (d->J < 1 || d->J > PPF_MAX_J || d->F < 1 || d->T < 1 || d->U < 1) return PPF_EINVAL;
  int rc = check_model(d->model);
  if (rc) return rc;
  if (!d->swarm_in || !d->swarm_out || !d->rw_sig || !d->rw_sig0 || !d->cool || !d->cool0) return PPF_EINVAL;
  if (d->swarm_in == d->swarm_out) return PPF_EINVAL;
  if (!d->ys || !d->loglik) return PPF_EINVAL;
  if (!(d->flags & PPF_F_INJECT) && !d->seeds) return PPF_EINVAL;
  if ((d->flags & PPF_F_INJECT) && (!d->inj_z || !d->inj_u || !d->inj_zp0 || !d->inj_zp)) return PPF_EINVAL;
  if ((d->flags & PPF_F_INJECT) && d->model.kind == PPF_MODEL_LG && !d->inj_z0) return PPF_EINVAL;
  if (d->model.kind == PPF_MODEL_RICKER && !d->ycon) return PPF_EINVAL;
  if ((d->flags & PPF_F_CLL) && !d->cll) return PPF_EINVAL;
  if ((d->flags & PPF_F_SAVE_ANC) && !d->anc) return PPF_EINVAL;
  return PPF_OK;
}

static void fill_if2(const ppf_perfilter_desc* d, Args& a) {
  ppf_pfilter_desc p;
  memset(&p, 0, sizeof(p));
  p.model = d->model;
  p.J = d->J; p.F = d->F; p.T = d->T; p.U = d->U;
  p.flags = (d->flags & (PPF_F_INJECT | PPF_F_CLL | PPF_F_SAVE_ANC | PPF_F_NO_CLUSTER)) |
            ((d->flags & PPF_F_NATURAL) ? 0u : PPF_F_EST);
  p.thresh = d->thresh;
  p.ys = d->ys; p.ycon = d->ycon; p.unit = d->unit; p.T_u = d->T_u;
  p.seeds = d->seeds; p.inj_z0 = d->inj_z0; p.inj_z = d->inj_z; p.inj_u = d->inj_u;
  p.loglik = d->loglik; p.cll = d->cll; p.anc = d->anc;
  fill_args(&p, a, MODE_IF2);
  a.swarm_in = d->swarm_in; a.swarm_out = d->swarm_out;
  a.rw_sig = d->rw_sig; a.rw_sig0 = d->rw_sig0; a.cool = d->cool; a.cool0 = d->cool0;
  a.inj_zp0 = d->inj_zp0; a.inj_zp = d->inj_zp;
}

// ---------------------------------------------------------------------------
// CUDA graphs (PPF_F_GRAPH): the launch sequence of a call is captured once
// and replayed for byte-identical descriptors.
// ---------------------------------------------------------------------------
constexpr int kGraphCap = 16;
constexpr size_t kGraphKeyMax = 512;
struct GraphEntry {
  unsigned char key[kGraphKeyMax];
  size_t klen;
  int dev;
  cudaGraphExec_t exec;
};
static GraphEntry g_graphs[kGraphCap];
static int g_graph_n = 0, g_graph_next = 0;

template <class Fn>
static int run_graphed(const void* key, size_t klen, cudaStream_t s, Fn&& launch) {
  if (klen > kGraphKeyMax || g_prof.enabled) return launch(s);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return PPF_ECUDA;
  if (cs != cudaStreamCaptureStatusNone) return launch(s);   // the caller is capturing
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PPF_ECUDA;
  for (int i = 0; i < g_graph_n; ++i) {
    GraphEntry& e = g_graphs[i];
    if (e.dev == dev && e.klen == klen && memcmp(e.key, key, klen) == 0)
      return cudaGraphLaunch(e.exec, s) == cudaSuccess ? PPF_OK : PPF_ECUDA;
  }
  // capture on a private stream (the caller's may be the legacy default
  // stream, which cannot be captured); the graph is then launched on theirs
  static cudaStream_t cap_stream[64] = {nullptr};
  if (dev < 0 || dev >= 64) return launch(s);
  if (!cap_stream[dev] && cudaStreamCreateWithFlags(&cap_stream[dev], cudaStreamNonBlocking) != cudaSuccess)
    return PPF_ECUDA;
  cudaStream_t cst = cap_stream[dev];
  if (cudaStreamBeginCapture(cst, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return PPF_ECUDA;
  const int rc = launch(cst);
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(cst, &g);
  if (rc != PPF_OK || ec != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return rc != PPF_OK ? rc : PPF_ECUDA;
  }
  cudaGraphExec_t ex = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return PPF_ECUDA;
  int idx;
  if (g_graph_n < kGraphCap) {
    idx = g_graph_n++;
  } else {                                   // full: replace the oldest entry
    idx = g_graph_next;
    g_graph_next = (g_graph_next + 1) % kGraphCap;
    cudaGraphExecDestroy(g_graphs[idx].exec);
  }
  GraphEntry& slot = g_graphs[idx];
  memcpy(slot.key, key, klen);
  slot.klen = klen;
  slot.dev = dev;
  slot.exec = ex;
  return cudaGraphLaunch(ex, s) == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

}  // namespace ppf

using namespace ppf;

extern "C" {

size_t ppf_pfilter_workspace_bytes(const ppf_pfilter_desc* d) {
  if (validate(d) != PPF_OK && !(d && d->J >= 1 && d->F >= 1)) return 0;
  Args a;
  fill_args(d, a, MODE_PF);
  return carve(a, choose_path(d), nullptr);
}

int ppf_pfilter(const ppf_pfilter_desc* d, void* stream) {
  int rc = validate(d);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Args a;
  fill_args(d, a, MODE_PF);
  const int path = choose_path(d);
  const size_t need = carve(a, path, nullptr);
  if (!d->workspace || d->ws_bytes < need) return PPF_EINVAL;
  carve(a, path, reinterpret_cast<unsigned char*>(d->workspace));
  auto launch = [&](cudaStream_t st) -> int {
    if (cudaMemsetAsync(d->workspace, 0, a.ctrl_bytes, st) != cudaSuccess) return PPF_ECUDA;
    if (path == PPF_PATH_STREAM) {
      // accumulators start at (max=-, min=+, nan=0)
      const int r = reset_accumulators(a, st);
      if (r) return r;
    }
    return run_pfilter_path(a, path, st);
  };
  if ((d->flags & PPF_F_GRAPH) && path != PPF_PATH_PLAIN) return run_graphed(d, sizeof(*d), s, launch);
  return launch(s);
}

size_t ppf_mop_workspace_bytes(const ppf_mop_desc* d) {
  if (!d || d->J < 1 || d->F < 1 || d->T < 1) return 0;
  ppf_pfilter_desc p;
  mop_to_pfilter(d, &p);
  Args a;
  fill_args(&p, a, MODE_MOP);
  MopWork w;
  memset(&w, 0, sizeof(w));
  return carve_mop(a, w, d, nullptr);
}

// value = -sum_t ll_t: the forward accumulates +ll into `value`, then a tiny
// kernel negates it (same stream).
__global__ void k_negate(double* v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = -v[i];
}

int ppf_mop(const ppf_mop_desc* d, void* stream) {
  int rc = validate_mop(d);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  ppf_pfilter_desc p;
  mop_to_pfilter(d, &p);
  Args a;
  fill_args(&p, a, MODE_MOP);
  a.flags |= PPF_F_SAVE_ANC;
  a.pwi = (d->flags & PPF_F_DPOP) ? d->process_weight_index : -1;
  MopWork w;
  memset(&w, 0, sizeof(w));
  const size_t need = carve_mop(a, w, d, nullptr);
  if (!d->workspace || d->ws_bytes < need) return PPF_EINVAL;
  carve_mop(a, w, d, reinterpret_cast<unsigned char*>(d->workspace));
  w.grad = d->grad;
  w.alpha = d->alpha;
  auto launch = [&](cudaStream_t st) -> int {
    if (cudaMemsetAsync(d->workspace, 0, a.ctrl_bytes, st) != cudaSuccess) return PPF_ECUDA;
    int r = reset_accumulators(a, st);
    if (r) return r;
    r = run_mop(a, w, st);
    if (r) return r;
    k_negate<<<(d->F + 127) / 128, 128, 0, st>>>(d->value, d->F);
    return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
  };
  if (d->flags & PPF_F_GRAPH) return run_graphed(d, sizeof(*d), s, launch);
  return launch(s);
}

size_t ppf_perfilter_workspace_bytes(const ppf_perfilter_desc* d) {
  if (!d || d->J < 1 || d->F < 1 || d->T < 1 || n_params_of(d->model) < 1) return 0;
  Args a;
  fill_if2(d, a);
  a.model.n_params = n_params_of(d->model);
  return carve_if2(a, nullptr);
}

int ppf_perfilter(const ppf_perfilter_desc* d, void* stream) {
  int rc = validate_if2(d);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Args a;
  fill_if2(d, a);
  const size_t need = carve_if2(a, nullptr);
  if (!d->workspace || d->ws_bytes < need) return PPF_EINVAL;
  carve_if2(a, reinterpret_cast<unsigned char*>(d->workspace));
  auto launch = [&](cudaStream_t st) -> int {
    if (cudaMemsetAsync(d->workspace, 0, a.ctrl_bytes, st) != cudaSuccess) return PPF_ECUDA;
    const int r = reset_accumulators(a, st);
    if (r) return r;
    return run_if2(a, st);
  };
  if (d->flags & PPF_F_GRAPH) return run_graphed(d, sizeof(*d), s, launch);
  return launch(s);
}

// grad[f][p] *= dvalue[f]
__global__ void k_scale_rows(double* g, const double* dv, int F, int P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < F * P) g[i] *= dv[i / P];
}

int ppf_mop_backward(const ppf_mop_desc* d, const double* dvalue, void* stream) {
  int rc = validate_mop(d);
  if (rc) return rc;
  if (!d->grad) return PPF_EINVAL;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  ppf_pfilter_desc p;
  mop_to_pfilter(d, &p);
  Args a;
  fill_args(&p, a, MODE_MOP);
  a.flags |= PPF_F_SAVE_ANC;
  a.pwi = (d->flags & PPF_F_DPOP) ? d->process_weight_index : -1;
  MopWork w;
  memset(&w, 0, sizeof(w));
  const size_t need = carve_mop(a, w, d, nullptr);
  if (!d->workspace || d->ws_bytes < need) return PPF_EINVAL;
  carve_mop(a, w, d, reinterpret_cast<unsigned char*>(d->workspace));
  w.grad = d->grad;
  w.alpha = d->alpha;
  rc = run_mop_backward(a, w, s);
  if (rc) return rc;
  if (dvalue) {
    const int n = d->F * d->model.n_params;
    k_scale_rows<<<(n + 255) / 256, 256, 0, s>>>(d->grad, dvalue, d->F, d->model.n_params);
  }
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

int ppf_autotune(const ppf_pfilter_desc* d, void* stream, int* best_tile) {
  int rc = validate(d);
  if (rc) return rc;
  if (!best_tile) return PPF_EINVAL;
  if (choose_path(d) != PPF_PATH_STREAM) {
    *best_tile = 0;
    return PPF_OK;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  ppf_pfilter_desc t;
  memcpy(&t, d, sizeof(t));
  t.path = PPF_PATH_STREAM;
  if (t.T > 16) t.T = 16;   // a prefix of the time loop; the per-step cost does not depend on t
  t.T_u = nullptr;
  const int tiles[3] = {kTileLarge, kTileMid, kTileSmall};
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return PPF_ECUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return PPF_ECUDA; }
  float best_ms = 0.0f;
  int best = 0;
  for (int tile : tiles) {
    t.tile = tile;
    float ms = 0.0f;
    for (int rep = 0; rep < 2 && rc == PPF_OK; ++rep) {   // first run warms up, second is timed
      if (cudaEventRecord(e0, s) != cudaSuccess) rc = PPF_ECUDA;
      if (!rc) rc = ppf_pfilter(&t, stream);
      if (!rc && cudaEventRecord(e1, s) != cudaSuccess) rc = PPF_ECUDA;
      if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = PPF_ECUDA;
      if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    }
    if (rc) break;
    if (!best || ms < best_ms) { best = tile; best_ms = ms; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  tune_store(d->model, d->J, d->F, d->U, (d->flags & PPF_F_INJECT) ? 1 : 0, best);
  *best_tile = best;
  return PPF_OK;
}

int ppf_simulate(const ppf_simulate_desc* d, void* stream) {
  if (!d) return PPF_EINVAL;
  if (d->F < 1 || d->F > 65535 || d->nsim < 1 || d->T < 0) return PPF_EINVAL;
  const int rc = check_model(d->model);
  if (rc) return rc;
  if (!d->theta || !d->seeds || !d->X || (d->T > 0 && !d->Y)) return PPF_EINVAL;
  return run_simulate(d, reinterpret_cast<cudaStream_t>(stream));
}

int ppf_workspace_status(const void* workspace, void* stream) {
  if (!workspace) return PPF_EINVAL;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  uint32_t err = 0;
  if (cudaMemcpyAsync(&err, workspace, sizeof(err), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PPF_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return PPF_ECUDA;
  if (err & 1u) return PPF_ETIMEOUT;
  if (err) return PPF_EINTERNAL;
  return PPF_OK;
}

long long ppf_debug_set_wait_limit(long long polls) {
  const long long prev = g_spin_cap;
  g_spin_cap = polls < 0 ? kSpinCap : (polls > kSpinCap ? kSpinCap : polls);
  return prev;
}

int ppf_profile_begin(void) {
  g_prof.enabled = true;
  g_prof.used = 0;
  return PPF_OK;
}

int ppf_profile_end(double* ms, int* count, int n) {
  if (!ms || !count || n < 1) return PPF_EINVAL;
  for (int i = 0; i < n; ++i) { ms[i] = 0.0; count[i] = 0; }
  for (int i = 0; i < g_prof.used; ++i) {
    if (cudaEventSynchronize(g_prof.evs[i].b) != cudaSuccess) return PPF_ECUDA;
    float t = 0.0f;
    cudaEventElapsedTime(&t, g_prof.evs[i].a, g_prof.evs[i].b);
    const int k = g_prof.evs[i].kind;
    if (k >= 0 && k < n) { ms[k] += t; count[k] += 1; }
  }
  g_prof.enabled = false;
  g_prof.used = 0;
  return PPF_OK;
}

const char* ppf_error_string(int code) {
  switch (code) {
    case PPF_OK: return "ok";
    case PPF_EINVAL: return "invalid argument";
    case PPF_ECUDA: return "CUDA launch or runtime error";
    case PPF_ETIMEOUT: return "a bounded device-side wait timed out";
    case PPF_EUNSUPPORTED: return "unsupported configuration";
    case PPF_EINTERNAL: return "a device-side consistency check failed";
    case PPF_ESCRATCH: return "the request needs more scratch than the no-allocation entry point holds";
    default: return "unknown error";
  }
}

const char* ppf_version(void) { return "ppf 0.1.0 sm_100a"; }

}  // extern "C"
