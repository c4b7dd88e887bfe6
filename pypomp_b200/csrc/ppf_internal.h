// ppf_internal.h -- host/device argument block shared by the kernels of
// libppf.so.  Not part of the public ABI (that is include/ppf.h).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <vector>
#include "ppf.h"

namespace ppf {

struct Acc;

enum { MODE_PF = 0, MODE_MOP = 1, MODE_IF2 = 2 };

constexpr size_t kResidentSmemMax = 220 * 1024;

// Everything a kernel needs, passed by value (well under the 32 KB limit).
struct Args {
  ppf_model model;
  int J, F, T, U;
  uint32_t flags;
  int mode;
  int pwi;          // DPOP: state component of the transition log-weight; -1 for MOP
  float thresh, logthresh;
  float base_init;  // log(1/J): the reference's initial log-weight (pfilter.py:35)
  float base_rs;    // -log(J): the log-weight after resampling (helpers.py:88-90)
  const float* theta;
  const float* ys;
  const float* ycon;
  const int* unit;
  const int* T_u;
  const uint64_t* seeds;
  const float* inj_z0;
  const float* inj_z;
  const float* inj_u;
  double* loglik;
  double* cll;
  float* ess;
  float* fmean;
  float* pmean;
  int* anc;
  float* logw;
  // workspace
  uint32_t* err;
  unsigned int* counter;  // [2]
  unsigned int* gbar;     // [3] grid barrier: arrivals, generation, abort (zeroed per call)
  uint64_t* slotw;        // [6][kInboxWords] per-CTA step inboxes of the grid-resident MOP
                          // forward (zeroed by its launch)
  Acc* acc[2];            // [F] each
  uint64_t* desc[2];      // [F][ntiles] each
  uint64_t* excl;         // [F][ntiles]
  uint64_t* tot;          // [F]
  unsigned int* fdone[2]; // [F] each: tiles of the filter whose total is out (k_sum)
  uint64_t* runpre;       // [F][ntiles][TPB] exclusive prefix of each thread's run of q in its tile
  float* X[2];            // [F][dx][J] each
  float* W[2];            // [F][J] each
  unsigned char* consts;  // [F][512 B] per-filter model constants
  int tile, ntiles;
  long long spin_cap;     // polls before a bounded device-side wait gives up
  size_t ctrl_bytes;      // leading workspace bytes zeroed per call
  // plain path
  uint64_t* pl_cdf;       // [J]
  uint64_t* pl_bsum;      // [nblk]
  uint64_t* pl_boff;      // [nblk]
  int* pl_anc;            // [J]
  int* pl_carry_dev;      // [1]
  // MOP forward saves (stream path, MODE_MOP): first-child offsets, state
  // checkpoints every ckpt_every steps, per-step max and weight sum of m.
  int* mop_off;           // [F][T][J+1]
  float* mop_ckpt;        // [F][nseg][DX][J]
  int ckpt_every, nseg;
  float* mop_M;           // [F][T]
  double* mop_S;          // [F][T]
  // IF2 perturbed filter (MODE_IF2): per-particle parameter swarm
  const float* swarm_in;  // [F][P][J] estimation scale
  float* swarm_out;       // [F][P][J] after the final resampling
  float* TH[2];           // [F][P][J] each, perturbed parameters of the live swarm
  const float* rw_sig;    // [P] per-step sds
  const float* rw_sig0;   // [P] t0 sds
  const float* cool;      // [U][T] cooling factor of the perturbation before step t
  const float* cool0;     // [U] cooling factor of the t0 perturbation
  const float* inj_zp0;   // [F][J][P] t0 perturbation normals (PPF_F_INJECT)
  const float* inj_zp;    // [F][T][J][P] per-step perturbation normals (PPF_F_INJECT)
  // host copies for host-side loops (plain path)
  const int* T_u_host;
  const int* unit_host;
};

enum { KIND_INIT = 0, KIND_SUM = 1, KIND_RESPROP = 2, KIND_RESIDENT = 3, KIND_PLAIN = 4,
       KIND_MOP_FWD = 5, KIND_MOP_RECOMP = 6, KIND_MOP_BWD = 7, KIND_IF2 = 8, KIND_CLUSTER = 9, KIND_SIMULATE = 10,
       KIND_COUNT = 16 };

struct Profiler {
  struct Ev { cudaEvent_t a, b; int kind; };
  bool enabled = false;
  int used = 0;
  std::vector<Ev> evs;
  void mark(int kind, cudaStream_t s, bool start);
};
extern Profiler g_prof;
#define PROF_BEGIN(kind) ::ppf::g_prof.mark(kind, s, true)
#define PROF_END(kind) ::ppf::g_prof.mark(kind, s, false)

// MOP adjoint working set (workspace carve-outs) and outputs.
struct MopWork {
  float* lx;      // [2][F][DX][J]
  float* lw;      // [2][F][J]
  float* sb;      // [F][ckpt_every][DX][J] recomputed states of one segment
  float* sb2;     // second segment buffer (persistent adjoint: two segments in flight)
  double* gpart;  // [F * ceil(J/256)][64] per-CTA gradient sums (persistent adjoint)
  double* gnat;   // [F][64] natural-scale gradient sums
  double* grad;   // out [F][P] estimation-scale gradient, or nullptr
  float alpha;
};

int run_pfilter_path(Args& a, int path, cudaStream_t s);
// the per-filter model constants (k_prep), dispatched by model
int run_prep(Args& a, cudaStream_t s);
// the streaming path with PPF_F_FAST (ppf_fast.cu, compiled with contraction)
int run_stream_fast(Args& a, cudaStream_t s);
int run_stream_any(Args& a, cudaStream_t s);   // stream path, any model
// Stream-path tile configurations (particles per CTA = threads x items per
// thread): the tile sets how many CTAs one step launches, F x ceil(J / tile).
constexpr int kTileLarge = 2048;   // 256 threads x 8
constexpr int kTileMid = 512;      // 128 threads x 4
constexpr int kTileSmall = 256;    // 64 threads x 4
constexpr int kNumSMs = 148;
// the wide LG instantiations (dx or dy above 4, up to 9)
inline bool lg_wide(const ppf_model& m) { return m.kind == PPF_MODEL_LG && (m.dx > 4 || m.dy > 4); }
// natural-scale gradient entries per filter in the MOP workspace: the padded
// layout of the largest model, LG 9 x 9 (81 + 81 + 45 + 45 + 9 = 261)
constexpr int kMaxNG = 264;
// CTAs of a grid-resident launch that publish per-step words (8 per SM)
constexpr int kMaxGridSlots = 8 * kNumSMs;
// words of one inbox array of the grid-resident MOP forward: F x C x C for F
// filters of C CTAs (C = 148 for one filter on one CTA per SM)
constexpr int kInboxWords = 32768;

int run_mop(Args& a, const MopWork& w, cudaStream_t s);
int run_mop_backward(Args& a, const MopWork& w, cudaStream_t s);
int run_if2(Args& a, cudaStream_t s);
// cluster-resident filters (ppf_cluster.cu): whether a cluster plan exists for
// this shape, and the launch
bool cluster_fits(const Args& a, bool if2);
int run_cluster(Args& a, bool if2, cudaStream_t s);
// Trajectories of the built-in models (ppf_simulate.cu); the descriptor is validated.
int run_simulate(const ppf_simulate_desc* d, cudaStream_t s);
int reset_accumulators(Args& a, cudaStream_t s);
size_t resident_smem_bytes(const Args& a);

}  // namespace ppf
