// ppf_mop.cu -- MOP-alpha objective and its hand-written adjoint.
//
// Replaces _mop_internal / _mop_step (pypomp/core/algorithms/mop.py:19-135)
// and the reverse-mode jax.value_and_grad of it (ad_helpers.py:32-54) that
// train uses (train.py:87-102).
//
// Forward: the stream particle filter in MOP mode -- resampling weights are
// the measurement densities m alone (mop.py:120, normalize(stop_gradient(m)))
// and the value is -sum_t [LSE(m_t) - log J] (with uniform carried weights
// LSE(wP + m) - LSE(wP) reduces to that).  It also keeps, per step, the
// ancestors, each parent's first-child offset, max m and sum exp(m - max),
// and the resampled states every `ckpt_every` steps (sqrt(T) by default).
//
// Adjoint, segment by segment from the last: states of the segment are
// recomputed from its checkpoint through the stored ancestors with the same
// Philox counters (bit-identical to the forward), then steps are swept
// backwards.  For slot j at step t (pi = softmax(m_t), g = -1):
//   Lx_j, Lw_j = sums of the adjoints of j's children (a contiguous range)
//   lm = Lw_j + g pi_j        (m enters LSE and the carried weight)
//   lwP = Lw_j + g (pi_j - 1/J)
//   lx(x^P) = Lx_j + lm dm/dx ; dtheta += lm dm/dtheta + lx dx^P/dtheta
//   adjoint of x^F_{t-1}[j] = (dx^P/dx)^T lx ; of wF_{t-1}[j] = alpha lwP
// and finally dtheta += (d rinit / dtheta)^T adjoint(x^F_{-1}).  The sums over
// children read the stored offsets, so they are deterministic.  DPOP
// (PPF_F_DPOP) has the same forward; its adjoint adds lwP to lx[pwi] before
// the model step (the transition log-weight rides on the carried weight).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "ppf.h"
#include "ppf_core.cuh"
#include "ppf_internal.h"
#include "ppf_kernels.cuh"
#include "ppf_models.cuh"
#include "ppf_stream.cuh"

namespace ppf {



struct MopBwd {
  const float* xin;    // x^F_{t-1} of filter 0: [DX][J], filter stride xin_fs
  size_t xin_fs;
  float* xout;         // recompute output x^F_t of filter 0, filter stride xout_fs
  size_t xout_fs;
  const float* lx_in;  // adjoint of x^F_t   [F][DX][J]
  const float* lw_in;  // adjoint of wF_t    [F][J]
  float* lx_out;       // adjoint of x^F_{t-1}
  float* lw_out;       // adjoint of wF_{t-1}
  double* gnat;        // [F][kMaxNG] natural-scale gradient
  float alpha;
};

template <class M, bool INJ>
__device__ __forceinline__ void particle_normals(const Args& a, int f, int j, int s, int n, float* z) {
  if (n <= 0) return;
  if (INJ) {
    const float* src = (s == 0) ? a.inj_z0 + ((size_t)f * a.J + j) * n
                                : a.inj_z + (((size_t)f * a.T + (s - 1)) * a.J + j) * n;
    for (int i = 0; i < n; ++i) z[i] = src[i];
  } else {
    pp_normals(a.seeds[f], (uint32_t)j, (uint32_t)s, PPF_TAG_PROCESS, n, z);
  }
}

// DPOP (dpop.py:203-209): the predicted state's component pwi is added to the
// carried weights as pw - stop_gradient(pw), so its adjoint is the carried
// weight's, lwP.  Added to the state adjoint before the model's backward step
// takes it through rproc; a no-op for MOP (pwi < 0).
template <int DX>
__device__ __forceinline__ void add_process_weight(float* lx, int pwi, float lwP) {
#pragma unroll
  for (int d = 0; d < DX; ++d)
    if (d == pwi) lx[d] += lwP;
}

// x^F_t[k] = rproc(x^F_{t-1}[anc_t[k]]) with the parent's noise.
template <class M, int TPB, bool INJ>
__global__ void __launch_bounds__(TPB) k_mop_recomp(Args a, MopBwd mb, int t) {
  __shared__ typename M::Consts c;
  constexpr int DX = M::MAXDX;
  const int f = blockIdx.y;
  if (t >= filter_len(a, filter_unit(a, f))) return;
  load_consts<M>(a, f, c);
  __syncthreads();
  const int J = a.J;
  const int k = blockIdx.x * TPB + threadIdx.x;
  if (k >= J) return;
  const int j = a.anc[((size_t)f * a.T + t) * J + k];
  const float* xin = mb.xin + f * mb.xin_fs;
  float x[DX];
#pragma unroll
  for (int d = 0; d < DX; ++d) x[d] = xin[d * J + j];
  float z[M::NZ];
  particle_normals<M, INJ>(a, f, j, t + 1, M::NZ, z);
  M::rproc(c, x, z);
  float* xo = mb.xout + f * mb.xout_fs;
#pragma unroll
  for (int d = 0; d < DX; ++d) xo[d * J + k] = x[d];
}

template <int TPB, int NG>
__device__ __forceinline__ void reduce_grad(const float* g, double* out, double* sd) {
#pragma unroll 1
  for (int i = 0; i < NG; ++i) {
    const double v = block_sum_f64<TPB>((double)g[i], sd);
    if (threadIdx.x == 0 && v != 0.0) atomicAdd(out + i, v);
  }
}

template <class M, int TPB, bool INJ>
__global__ void __launch_bounds__(TPB) k_mop_bwd(Args a, MopBwd mb, int t) {
  __shared__ typename M::Consts c;
  __shared__ double sd[TPB / 32];
  constexpr int DX = M::MAXDX;
  const int f = blockIdx.y;
  const int u = filter_unit(a, f);
  if (t >= filter_len(a, u)) return;
  load_consts<M>(a, f, c);
  __syncthreads();
  const typename M::Consts cr = c;
  const int J = a.J;
  Obs<M> ob;
  ob.load(a, u, t);
  float g[M::NG];
#pragma unroll
  for (int i = 0; i < M::NG; ++i) g[i] = 0.0f;
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j < J) {
    const float* xin = mb.xin + f * mb.xin_fs;
    float x[DX];
#pragma unroll
    for (int d = 0; d < DX; ++d) x[d] = xin[d * J + j];
    float z[M::NZ];
    particle_normals<M, INJ>(a, f, j, t + 1, M::NZ, z);
    typename M::Keep kp;
    const float m = M::fwd_keep(cr, ob.y, ob.yc, x, z, kp);
    const float Mt = a.mop_M[(size_t)f * a.T + t];
    const double S1 = a.mop_S[(size_t)f * a.T + t];
    float pi = 0.0f;
    if (S1 > 0.0 && m == m) pi = (float)((double)pp_expf(m - Mt) / S1);
    // adjoints of j's children (contiguous range of step t)
    const int* off = a.mop_off + ((size_t)f * a.T + t) * (J + 1);
    const int lo = off[j], hi = off[j + 1];
    float lx[DX];
#pragma unroll
    for (int d = 0; d < DX; ++d) lx[d] = 0.0f;
    float lw = 0.0f;
    const float* lxi = mb.lx_in + (size_t)f * DX * J;
    const float* lwi = mb.lw_in + (size_t)f * J;
    // a parent of many children (degenerate weights): several loads in flight,
    // the sums still taken in child order
#pragma unroll 4
    for (int k = lo; k < hi; ++k) {
#pragma unroll
      for (int d = 0; d < DX; ++d) lx[d] += lxi[d * J + k];
      lw += lwi[k];
    }
    const float gl = -1.0f;                       // d(-sum ll)/d ll_t
    const float lm = lw + gl * pi;
    const float lwP = lw + gl * (pi - 1.0f / (float)J);
    if (m == m && m > -INFINITY) {
      add_process_weight<DX>(lx, a.pwi, lwP);
      M::bwd(cr, x, z, kp, lm, lx, g);
    } else {
#pragma unroll
      for (int d = 0; d < DX; ++d) lx[d] = 0.0f;
    }
    float* lxo = mb.lx_out + (size_t)f * DX * J;
#pragma unroll
    for (int d = 0; d < DX; ++d) lxo[d * J + j] = lx[d];
    mb.lw_out[(size_t)f * J + j] = mb.alpha * lwP;
  }
  reduce_grad<TPB, M::NG>(g, mb.gnat + (size_t)f * kMaxNG, sd);
}

// dtheta += (d rinit / dtheta)^T adjoint(x^F_{-1})
template <class M, int TPB, bool INJ>
__global__ void __launch_bounds__(TPB) k_mop_bwd_init(Args a, MopBwd mb) {
  __shared__ typename M::Consts c;
  __shared__ double sd[TPB / 32];
  constexpr int DX = M::MAXDX;
  const int f = blockIdx.y;
  load_consts<M>(a, f, c);
  __syncthreads();
  const int J = a.J;
  float g[M::NG];
#pragma unroll
  for (int i = 0; i < M::NG; ++i) g[i] = 0.0f;
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j < J) {
    float z0[M::NZ0 > 0 ? M::NZ0 : 1];
    particle_normals<M, INJ>(a, f, j, 0, M::NZ0, z0);
    float lx0[DX];
    const float* lxi = mb.lx_in + (size_t)f * DX * J;
#pragma unroll
    for (int d = 0; d < DX; ++d) lx0[d] = lxi[d * J + j];
    M::bwd_init(c, z0, lx0, g);
  }
  reduce_grad<TPB, M::NG>(g, mb.gnat + (size_t)f * kMaxNG, sd);
}

// Canonical-order gradient from the natural-scale sums, chained to the
// estimation scale unless the parameters are given on the natural scale.
template <class M>
struct Chain;

template <int DX, int DYS, int MDY>
struct Chain<LG<DX, DYS, MDY>> {
  using L = LG<DX, DYS, MDY>;
  __device__ static double map(const ppf_model& m, const float* th, const double* gn, int p, bool est) {
    const int dy = m.dy;
    const int nA = DX * DX, nC = dy * DX, nQ = DX * (DX + 1) / 2, nR = dy * (dy + 1) / 2;
    if (p < nA) return gn[L::GA + p];
    p -= nA;
    if (p < nC) return gn[L::GC + p];
    p -= nC;
    if (p < nQ) {
      double v = gn[L::GQ + p];
      for (int i = 0; i < DX; ++i)
        if (est && p == i * (i + 1) / 2 + i) v *= (double)pp_expf(th[nA + nC + p]);
      return v;
    }
    p -= nQ;
    if (p < nR) {
      double v = gn[L::GR + p];
      for (int i = 0; i < dy; ++i)
        if (est && p == i * (i + 1) / 2 + i) v *= (double)pp_expf(th[nA + nC + nQ + p]);
      return v;
    }
    p -= nR;
    return gn[L::GX0 + p];
  }
};
template <>
struct Chain<SV> {
  __device__ static double map(const ppf_model&, const float* th, const double* gn, int p, bool est) {
    if (!est) return gn[p];
    if (p < 3) return gn[p] * (double)pp_expf(th[p]);
    if (p == 3) {
      const double r = (double)pp_tanhf_det(th[3]);
      return gn[3] * (1.0 - r * r);
    }
    return gn[p];
  }
};
template <>
struct Chain<Ricker> {
  __device__ static double map(const ppf_model&, const float* th, const double* gn, int p, bool est) {
    return est ? gn[p] * (double)pp_expf(th[p]) : gn[p];
  }
};

template <class M>
__global__ void k_mop_chain(Args a, const double* gnat, double* grad) {
  const int f = blockIdx.x;
  const int P = a.model.n_params;
  for (int p = threadIdx.x; p < P; p += blockDim.x)
    grad[(size_t)f * P + p] = Chain<M>::map(a.model, a.theta + (size_t)f * P, gnat + (size_t)f * kMaxNG, p,
                                            (a.flags & PPF_F_EST) != 0);
}

// ---------------------------------------------------------------------------
// Persistent form: the whole forward in one cooperative launch and the whole
// adjoint sweep in another, with grid barriers between the steps instead of
// kernel boundaries.  For few filters of up to ~10^5 particles a step is a
// few microseconds of work, and two launches per step (plus the adjoint's
// two) cost more than the work; here the per-step cost is the barriers.
//
// Forward: CTA v owns tile (f, b) = (v / ntiles, v % ntiles) and runs the
// streaming kernels' own tile bodies (init_tile, sum_tile, resprop_tile) in
// sequence: the results are bit-identical to the per-step launches.
//
// Adjoint: the CTAs of filter f stride over its particles.  Segments are
// swept from the last, as in mop_backward, but the recomputation of segment
// s-1 runs in the same barrier intervals as the adjoint steps of segment s
// (two segment buffers), so the sweep costs one barrier per step.  Each
// thread sums its gradient terms in float over a segment, then the warp adds
// them into per-warp float64 sums; the per-CTA totals are added in CTA order
// by k_mop_chain_parts, so the gradient does not depend on scheduling.
// ---------------------------------------------------------------------------

struct MopBwdP {
  float* sb[2];     // [F][L][DX][J] each: recomputed states of one segment
  float* lx;        // [2][F][DX][J] adjoint of x^F by step parity
  float* lw;        // [2][F][J]     adjoint of wF by step parity
  double* gpart;    // [gridDim.x][kMaxNG] per-CTA natural-scale gradient sums
  float alpha;
  int nbf;          // CTAs per filter
};

template <class M, int N, bool INJ>
__device__ __forceinline__ void own_normals(const Args& a, int f, int j, int s, float* z) {
  if (N <= 0) return;
  if (INJ) {
    const float* src = (s == 0) ? a.inj_z0 + ((size_t)f * a.J + j) * N
                                : a.inj_z + (((size_t)f * a.T + (s - 1)) * a.J + j) * N;
#pragma unroll
    for (int i = 0; i < N; ++i) z[i] = src[i];
  } else {
    pp_normals_own(a.seeds[f], (uint32_t)j, (uint32_t)s, PPF_TAG_PROCESS, N, z);
  }
}

template <class M, int TPB, int IT, bool INJ>
__global__ void __launch_bounds__(TPB) k_mop_fwd_persist(Args a, GridBar gb) {
  const int f = blockIdx.x / a.ntiles, b = blockIdx.x % a.ntiles;
  init_tile<M, TPB, INJ>(a, f, b);
  if (!grid_sync(gb)) return;
  for (int t = 0; t < a.T; ++t) {
    sum_tile<M, TPB, IT, false>(a, t, f, b);
    if (!grid_sync(gb)) return;
    if (t < filter_len(a, filter_unit(a, f))) tile_prefix(a, t, f, b);
    resprop_tile<M, TPB, IT, INJ, false>(a, t, f, b);
    if (!grid_sync(gb)) return;
  }
}

// ---------------------------------------------------------------------------
// Grid-resident MOP forward: one cooperative launch for the whole time loop,
// C CTAs per filter, CTA c owning particles [c JC, (c+1) JC) (the structure
// of the cluster kernel, ppf_cluster.cu, at grid scope).  CTAs of one filter
// exchange their per-step numbers through tagged words in global memory
// instead of grid barriers: each CTA publishes one word per quantity and step
// (tag = step + 1 in the top 12 bits), and a reader's bounded poll of the C
// words of its filter is both the exchange and the wait.  Per observation t:
//   A. read the max / min / NaN words of the weights produced for t (the
//      release that published them also publishes those children's states and
//      weights), load the CTA's slice of parents from global memory into shared
//      memory (at t = 0 the initial states are already there), form their
//      fixed-point weights, block-scan them and publish the slice total;
//   B. read the C slice totals: this slice's exclusive prefix and the filter
//      total; first-child offsets of the slice's parents; one child per thread
//      at a time: rproc + dmeas, the child's state and weight written to global
//      memory, its ancestor, the first-child offsets and checkpoints kept for
//      the adjoint; then publish the max / min / NaN of the weights produced.
// Arithmetic, Philox counters and the order of the float64 log-likelihood sum
// are the streaming kernels', so results are bit-identical to them.  Words
// are double-buffered by step parity: a CTA can be at most one phase ahead of
// any other CTA of its filter, so a word is never overwritten before every
// reader has seen it (the argument is spelled out at the poll sites).
// ---------------------------------------------------------------------------

constexpr int kGridTagShift = 52;
constexpr int kGridMaxC = 256;          // CTAs per filter (8 words per polling lane)

__device__ __forceinline__ uint64_t grid_word(int tag, uint64_t v) {
  return ((uint64_t)((unsigned)tag & 0xfffu) << kGridTagShift) | v;
}

// Warp 0: read the C words of this CTA's inbox w[0..C) (word r is written by
// CTA r of the filter, and no other CTA reads this inbox), re-reading each
// word until it carries the step's tag (lane r polls words r, r + 32, ...),
// then combine the values with fn(r, value).  A word seen with its tag is not
// read again: no writer reuses its slot before this CTA has moved on (the
// argument is at the call sites).  The polls are relaxed; the acquire fence
// after the last one orders the CTA's later reads after every writer's
// release of its word (the CTA barrier that follows extends this to the
// other warps).  The wait is bounded: after spin_cap rounds, or when another
// CTA aborted, lane 0 sets the error and abort words and all of warp 0
// returns false.
template <class Fn>
__device__ __forceinline__ bool grid_gather(const uint64_t* w, int C, int tag, const Args& a, Fn fn) {
  constexpr int PER = kGridMaxC / 32;
  const int lane = threadIdx.x & 31;
  unsigned int* abortw = a.gbar + 2;
  const uint64_t want = (uint64_t)((unsigned)tag & 0xfffu);
  const uint64_t vm = (1ull << kGridTagShift) - 1;
  uint64_t v[PER];
  unsigned int need = 0u;   // bit i: word lane + 32 i not yet seen with the tag
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    v[i] = 0ull;
    if (lane + 32 * i < C) need |= 1u << i;
  }
  long long spins = 0;
  for (;;) {
    // all of a round's loads are issued before any of them is examined, so a
    // round costs one memory round trip, not one per word
    const unsigned int nd = need;
    uint64_t r[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i)
      if (nd & (1u << i)) r[i] = ld_relaxed_u64(w + lane + 32 * i);
#pragma unroll
    for (int i = 0; i < PER; ++i)
      if (nd & (1u << i)) {
        v[i] = r[i];
        if ((r[i] >> kGridTagShift) == want) need &= ~(1u << i);
      }
    if (!__any_sync(0xffffffffu, need != 0u)) break;
    int stop = 0;
    if (lane == 0) stop = (++spins > a.spin_cap) || ld_relaxed_u32(abortw) != 0u;
    stop = __shfl_sync(0xffffffffu, stop, 0);
    if (stop) {
      if (lane == 0) {
        atomicOr(a.err, 1u);
        atomicExch(abortw, 1u);
      }
      return false;
    }
  }
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
#pragma unroll
  for (int i = 0; i < PER; ++i)
    if (lane + 32 * i < C) fn(lane + 32 * i, v[i] & vm);
  return true;
}

template <class M, int TPB, bool INJ>
__global__ void __launch_bounds__(TPB, 1) k_mop_fwd_grid(Args a, int C, int JC) {
  constexpr int DX = M::MAXDX;
  constexpr int NW = TPB / 32;
  constexpr int ITM = 4;                 // parents per thread at most (JC <= 4 TPB)
  extern __shared__ __align__(16) float smf[];
  __shared__ typename M::Consts csh;
  __shared__ uint64_t s_scan[NW + 1];
  __shared__ unsigned int smk[3 * NW];
  __shared__ unsigned int s_key[3];      // max key, min key, NaN of the filter's weights
  __shared__ uint64_t s_sum[2];          // exclusive prefix of this slice, filter total
  __shared__ int s_ok;

  const int f = blockIdx.x / C, c = blockIdx.x % C;
  const int u = filter_unit(a, f);
  const int Tf = filter_len(a, u);
  const int J = a.J, T = a.T, L = a.ckpt_every;
  const int base = c * JC;
  const int nc = max(0, min(JC, J - base));
  // Inboxes: per quantity (max, min, sum) and step parity, an array of
  // [F][C readers][C writers] words.  A CTA pushes its word into every inbox
  // of its filter and polls only its own, so the polling of one CTA does not
  // contend with that of the others.
  const size_t box = (size_t)gridDim.x * C;
  uint64_t* maxw[2] = {a.slotw, a.slotw + box};
  uint64_t* minw[2] = {a.slotw + 2 * box, a.slotw + 3 * box};
  uint64_t* sumw[2] = {a.slotw + 4 * box, a.slotw + 5 * box};
  const size_t fin = (size_t)f * C * C;  // this filter's inboxes
  const size_t mine = fin + (size_t)c * C;   // this CTA's inbox
  // with no resampling threshold (MOP: always resample) the min key is not needed
  const bool need_min = a.logthresh != -INFINITY;
  float* Xs = smf;                       // [DX][JC] parents of the current step
  float* Ws = Xs + DX * JC;              // [JC]
  int* st = reinterpret_cast<int*>(Ws + JC);   // [JC + 4] first-child offsets
  const int ITC = (JC + TPB - 1) / TPB;  // parents per thread (contiguous), <= ITM
  const int l0 = threadIdx.x * ITC;
  const int l1 = min(l0 + ITC, nc);

  load_consts<M>(a, f, csh);
  __syncthreads();
  const typename M::Consts cr = csh;

  // block max / min / NaN of the weights this CTA produced, published for
  // step `tag - 1` after every thread's stores: the release store of the max
  // word publishes the children's states and weights with it
  auto publish_keys = [&](unsigned int mx, unsigned int mn, unsigned int nn, int par, int tag) {
    mx = warp_max_u32(mx);
    mn = warp_min_u32(mn);
    nn = __any_sync(0xffffffffu, nn != 0u) ? 1u : 0u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { smk[warp] = mx; smk[NW + warp] = mn; smk[2 * NW + warp] = nn; }
    __syncthreads();
    // thread r (r < C) combines the warps' numbers and pushes the word to CTA
    // r's inbox; each release store publishes the CTA's children with it
    // (every thread's stores precede the barrier above)
    for (int r = threadIdx.x; r < C; r += TPB) {
      unsigned int A = 0u, B = 0xffffffffu, O = 0u;
#pragma unroll
      for (int w = 0; w < NW; ++w) { A = max(A, smk[w]); B = min(B, smk[NW + w]); O |= smk[2 * NW + w]; }
      const size_t slot = fin + (size_t)r * C + c;
      if (need_min) st_relaxed_u64(minw[par] + slot, grid_word(tag, (uint64_t)B));
      st_release_u64(maxw[par] + slot, grid_word(tag, ((uint64_t)O << 32) | A));
    }
  };

  // ---- initial states into shared memory, propagated into observation 0
  {
    Obs<M> ob;
    ob.load(a, u, 0);
    float* logw0 = a.logw ? a.logw + (size_t)f * T * J : nullptr;
    unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
    for (int l = threadIdx.x; l < nc; l += TPB) {
      const int k = base + l;
      float x[DX];
      float z0[M::NZ0 > 0 ? M::NZ0 : 1];
      step_noise<M>(a, f, k, 0, M::NZ0, z0);
      M::rinit(cr, z0, x);
      if (a.mop_ckpt)
#pragma unroll
        for (int d = 0; d < DX; ++d) a.mop_ckpt[((size_t)f * a.nseg * DX + d) * J + k] = x[d];
      float z[M::NZ > 0 ? M::NZ : 1];
      step_noise<M>(a, f, k, 1, M::NZ, z);
      const float w = 0.0f + step1<M>(cr, ob, x, z);
#pragma unroll
      for (int d = 0; d < DX; ++d) Xs[d * JC + l] = x[d];
      Ws[l] = w;
      accum_maxmin(w, mx, mn, nn);
      if (logw0) logw0[k] = w;
    }
    publish_keys(mx, mn, nn, 0, 1);
  }

  double ll_acc = 0.0;
  for (int t = 0; t < Tf; ++t) {
    const int pc = t & 1, pn = pc ^ 1;
    const bool last = (t == Tf - 1);
    Obs<M> ob;
    if (!last) ob.load(a, u, t + 1);

    // A. The keys of step t's weights (tag t+1), written at the end of step
    //    t-1.  A CTA overwrites its key word (tag t+3) only at the end of step
    //    t+1, after gathering the step t+1 key words, which every CTA of the
    //    filter releases only after its own gather here.
    if (threadIdx.x < 32) {
      unsigned int A = 0u, B = 0xffffffffu, O = 0u;
      bool ok = grid_gather(maxw[pc] + mine, C, t + 1, a, [&](int, uint64_t v) {
        A = max(A, (unsigned int)v);
        O |= (unsigned int)(v >> 32);
      });
      if (ok && need_min)
        ok = grid_gather(minw[pc] + mine, C, t + 1, a, [&](int, uint64_t v) { B = min(B, (unsigned int)v); });
      A = warp_max_u32(A);
      B = warp_min_u32(B);
      O = __any_sync(0xffffffffu, O != 0u) ? 1u : 0u;
      if (threadIdx.x == 0) { s_key[0] = A; s_key[1] = need_min ? B : A; s_key[2] = O; s_ok = ok ? 1 : 0; }
    }
    // the systematic draw of step t does not depend on the exchange
    const uint32_t u32 = resample_u32(a, f, t);
    __syncthreads();
    if (!s_ok) return;
    Acc acc;                 // the fields this kernel's flags read (no ESS / means here)
    acc.pad = 0u;
    acc.s2 = 0.0;
    acc.maxkey = s_key[0];
    acc.minkey = s_key[1];   // (= max key when unused: decide_resample then depends on NaN only)
    acc.nan = s_key[2];
    const bool nanf = acc.nan != 0;
    const float Mx = keyf(acc.maxkey);
    const bool collapsed = !nanf && Mx == -INFINITY;
    const bool qc = nanf || Mx == -INFINITY;
    // parents of step t >= 1 were written to global memory by whichever CTAs
    // drew them (visible after the gather's acquire and the barrier): states
    // into shared memory for the children, each thread's own weights straight
    // into registers (and shared memory, for steps without resampling).  At
    // t = 0 they are already in shared memory.
    float wv[ITM];
    if (t > 0) {
      const float* Xg = a.X[pc] + (size_t)f * DX * J + base;
      const float* Wg = a.W[pc] + (size_t)f * J + base;
#pragma unroll
      for (int i = 0; i < ITM; ++i) wv[i] = (l0 + i < l1) ? Wg[l0 + i] : 0.0f;
      for (int l = threadIdx.x; l < nc; l += TPB)
#pragma unroll
        for (int d = 0; d < DX; ++d) Xs[d * JC + l] = Xg[(size_t)d * J + l];
#pragma unroll
      for (int i = 0; i < ITM; ++i)
        if (l0 + i < l1) Ws[l0 + i] = wv[i];
    } else {
#pragma unroll
      for (int i = 0; i < ITM; ++i) wv[i] = (l0 + i < l1) ? Ws[l0 + i] : 0.0f;
    }
    uint64_t q[ITM];
    uint64_t qs = 0;
#pragma unroll
    for (int i = 0; i < ITM; ++i) {
      q[i] = (l0 + i < l1) ? qweight(wv[i], Mx, qc) : 0ull;
      qs += q[i];
    }
    uint64_t btot;
    const uint64_t tex = block_excl_scan_u64_1b<TPB>(qs, s_scan, btot);
    // sum words of step t (tag t+1) overwrite those of step t-2: their readers
    // gathered them before releasing their step t key words, which this CTA
    // has gathered (the words carry values only, so the store is relaxed)
    for (int r = threadIdx.x; r < C; r += TPB)
      st_relaxed_u64(sumw[pc] + fin + (size_t)r * C + c, grid_word(t + 1, btot));

    // B. slice prefix and filter total
    if (threadIdx.x < 32) {
      uint64_t E = 0, tot = 0;
      const bool ok = grid_gather(sumw[pc] + mine, C, t + 1, a, [&](int r, uint64_t v) {
        tot += v;
        E += (r < c) ? v : 0ull;
      });
      E = warp_sum_u64(E);
      tot = warp_sum_u64(tot);
      if (threadIdx.x == 0) { s_sum[0] = E; s_sum[1] = tot; s_ok = ok ? 1 : 0; }
    }
    __syncthreads();
    if (!s_ok) return;
    const uint64_t E = s_sum[0], tot = s_sum[1];
    const bool rs = decide_resample(a, acc);
    float lt32 = 0.0f;
    if (rs) {
      const Offsets o = make_offsets(tot, u32, J);
      if (l0 < nc && !run_has_heavy(o, q)) {
        OffWalk wk = offwalk_init(o, E + tex);
        st[l0] = wk.k;
#pragma unroll
        for (int i = 0; i < ITM; ++i) {
          if (l0 + i >= l1) break;
          const int kn = offwalk_add(o, wk, q[i]);
          if (l0 + i + 1 < l1 || l0 + i + 1 == nc) st[l0 + i + 1] = kn;
        }
      } else if (l0 < nc) {
        uint64_t C = E + tex;   // a heavy parent in the run: closed form throughout
        st[l0] = nchild_fast(o, C);
#pragma unroll
        for (int i = 0; i < ITM; ++i) {
          if (l0 + i >= l1) break;
          C += q[i];
          const int kn = nchild_fast(o, C);
          if (l0 + i + 1 < l1 || l0 + i + 1 == nc) st[l0 + i + 1] = kn;
        }
      }
    } else {
      if (nanf) lt32 = __int_as_float(0x7fc00000);
      else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
      for (int l = l0; l < l1; ++l) st[l] = base + l;
      if (l0 < nc && l1 == nc) st[nc] = base + nc;
    }
    __syncthreads();
    if (a.mop_off) {
      int* off = a.mop_off + ((size_t)f * T + t) * (J + 1) + base;
      for (int l = threadIdx.x; l <= nc; l += TPB)
        if (l < nc || base + nc == J) off[l] = st[l];
    }
    float* ckpt = nullptr;
    if (a.mop_ckpt && (t + 1) % L == 0 && (t + 1) / L < a.nseg)
      ckpt = a.mop_ckpt + ((size_t)f * a.nseg + (t + 1) / L) * DX * J;
    unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
    if (nc > 0) {
      const int klo = st[0], khi = st[nc];
      const float nwc = -pp_logf((float)J);
      int* anc = a.anc ? a.anc + ((size_t)f * T + t) * J : nullptr;
      float* logw = (a.logw && !last) ? a.logw + ((size_t)f * T + t + 1) * J : nullptr;
      float* Xn = a.X[pn] + (size_t)f * DX * J;
      float* Wn = a.W[pn] + (size_t)f * J;
#pragma unroll 1
      for (int k = klo + (int)threadIdx.x; k < khi; k += TPB) {
        const int l = find_parent(st, nc, k);
        if (anc) anc[k] = base + l;
        float x[DX];
#pragma unroll
        for (int d = 0; d < DX; ++d) x[d] = Xs[d * JC + l];
        if (ckpt)
#pragma unroll
          for (int d = 0; d < DX; ++d) ckpt[(size_t)d * J + k] = x[d];
        if (last) continue;
        float z[M::NZ > 0 ? M::NZ : 1];
        step_noise<M>(a, f, k, t + 2, M::NZ, z);
        const float wb = rs ? 0.0f : (collapsed ? nwc : Ws[l] - lt32);
        const float w = wb + step1<M>(cr, ob, x, z);
        accum_maxmin(w, mx, mn, nn);
#pragma unroll
        for (int d = 0; d < DX; ++d) Xn[(size_t)d * J + k] = x[d];
        Wn[k] = w;
        if (logw) logw[k] = w;
      }
    }
    // keys of step t+1's weights (tag t+2) overwrite those of step t-1 (see A)
    if (!last) publish_keys(mx, mn, nn, pn, t + 2);
    // the step's log-likelihood term and saved per-step numbers, by a thread
    // outside warp 0 once the keys are out (off the exchange's critical path)
    if (c == 0 && threadIdx.x == TPB - 32) finalize_step(a, f, t, acc, tot, &ll_acc);
    // No barrier here: shared memory is next written after the barrier that
    // follows the next key gather, which every thread reaches only after its
    // reads of this step (publish_keys' barrier orders smk).
  }
  if (c == 0 && threadIdx.x == TPB - 32) a.loglik[f] = ll_acc;
}

template <class M, int TPB, bool INJ>
__global__ void __launch_bounds__(TPB) k_mop_bwd_persist(Args a, MopBwdP mb, GridBar gb) {
  constexpr int DX = M::MAXDX, NG = M::NG, NW = TPB / 32;
  constexpr int NZ = M::NZ > 0 ? M::NZ : 1, NZ0 = M::NZ0 > 0 ? M::NZ0 : 1;
  __shared__ typename M::Consts c;
  __shared__ double s_g[NW][NG];
  const int f = blockIdx.x / mb.nbf, cb = blockIdx.x % mb.nbf;
  const int u = filter_unit(a, f), Tf = filter_len(a, u);
  const int J = a.J, T = a.T, L = a.ckpt_every;
  load_consts<M>(a, f, c);
  for (int i = threadIdx.x; i < NW * NG; i += TPB) (&s_g[0][0])[i] = 0.0;
  __syncthreads();
  const int stride = mb.nbf * TPB;
  const int j0 = cb * TPB + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t sbf = (size_t)f * L * DX * J;
  const float* ckf = a.mop_ckpt + (size_t)f * a.nseg * DX * J;
  // Gradient terms: each particle-step's float terms are added into float64
  // per thread, as the per-step kernels add them across a block, for up to 32
  // entries (SV, Ricker, LG up to dx = dy = 2); the larger LG models sum a
  // segment's terms in float per thread before the float64 warp sums, to stay
  // within registers.
  constexpr bool GD = NG <= 32;
  float gs[NG];
  double gd[GD ? NG : 1];
#pragma unroll
  for (int i = 0; i < NG; ++i) gs[i] = 0.0f;
#pragma unroll
  for (int i = 0; i < (GD ? NG : 1); ++i) gd[i] = 0.0;
  auto fold = [&]() {       // one particle-step's terms into the float64 sums
    if (GD) {
#pragma unroll
      for (int i = 0; i < NG; ++i) {
        gd[i] += (double)gs[i];
        gs[i] = 0.0f;
      }
    }
  };

  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i < NG; ++i) {
      const double v = warp_sum_f64(GD ? gd[GD ? i : 0] : (double)gs[i]);
      if (lane == 0) s_g[warp][i] += v;
      gs[i] = 0.0f;
      if (GD) gd[GD ? i : 0] = 0.0;
    }
  };
  // x^F_{t-1} for step t of segment seg: its checkpoint, or the buffer
  auto xin_of = [&](int t, int seg, const float* sbuf) -> const float* {
    const int t0 = seg * L;
    return (t == t0) ? ckf + (size_t)seg * DX * J : sbuf + sbf + (size_t)(t - 1 - t0) * DX * J;
  };
  // x^F_t[k] = rproc(x^F_{t-1}[anc_t[k]]) with the parent's normals
  auto recompute = [&](int t, int seg, float* sbuf) {
    const float* xin = xin_of(t, seg, sbuf);
    float* xo = sbuf + sbf + (size_t)(t - seg * L) * DX * J;
    const int* anc = a.anc + ((size_t)f * T + t) * J;
    for (int k = j0; k < J; k += stride) {
      const int j = anc[k];
      float x[DX];
#pragma unroll
      for (int d = 0; d < DX; ++d) x[d] = xin[d * J + j];
      float z[NZ];
      own_normals<M, M::NZ, INJ>(a, f, j, t + 1, z);
      M::rproc(c, x, z);
#pragma unroll
      for (int d = 0; d < DX; ++d) xo[d * J + k] = x[d];
    }
  };
  // the adjoint step of k_mop_bwd for this thread's particles
  auto adjoint = [&](int t, int seg, const float* sbuf) {
    const float* xin = xin_of(t, seg, sbuf);
    Obs<M> ob;
    ob.load(a, u, t);
    const float Mt = a.mop_M[(size_t)f * T + t];
    const double S1 = a.mop_S[(size_t)f * T + t];
    const int* off = a.mop_off + ((size_t)f * T + t) * (J + 1);
    const int pin = t & 1, pout = pin ^ 1;
    const float* lxi = mb.lx + ((size_t)pin * a.F + f) * DX * J;
    const float* lwi = mb.lw + ((size_t)pin * a.F + f) * J;
    float* lxo = mb.lx + ((size_t)pout * a.F + f) * DX * J;
    float* lwo = mb.lw + ((size_t)pout * a.F + f) * J;
    for (int j = j0; j < J; j += stride) {
      float x[DX];
#pragma unroll
      for (int d = 0; d < DX; ++d) x[d] = xin[d * J + j];
      float z[NZ];
      own_normals<M, M::NZ, INJ>(a, f, j, t + 1, z);
      typename M::Keep kp;
      const float m = M::fwd_keep(c, ob.y, ob.yc, x, z, kp);
      float pi = 0.0f;
      if (S1 > 0.0 && m == m) pi = (float)((double)pp_expf(m - Mt) / S1);
      const int lo = off[j], hi = off[j + 1];
      float lx[DX];
#pragma unroll
      for (int d = 0; d < DX; ++d) lx[d] = 0.0f;
      float lw = 0.0f;
      // a parent of many children (degenerate weights): several loads in flight,
      // the sums still taken in child order
#pragma unroll 4
      for (int k = lo; k < hi; ++k) {
#pragma unroll
        for (int d = 0; d < DX; ++d) lx[d] += lxi[d * J + k];
        lw += lwi[k];
      }
      const float gl = -1.0f;
      const float lm = lw + gl * pi;
      const float lwP = lw + gl * (pi - 1.0f / (float)J);
      if (m == m && m > -INFINITY) {
        add_process_weight<DX>(lx, a.pwi, lwP);
        M::bwd(c, x, z, kp, lm, lx, gs);
        fold();
      } else {
#pragma unroll
        for (int d = 0; d < DX; ++d) lx[d] = 0.0f;
      }
#pragma unroll
      for (int d = 0; d < DX; ++d) lxo[d * J + j] = lx[d];
      lwo[j] = mb.alpha * lwP;
    }
  };

  {   // recompute the last segment before its sweep
    const int seg = a.nseg - 1, t0 = seg * L, t1 = min(t0 + L, T);
    for (int t = t0; t < t1 - 1; ++t) {
      if (t < Tf) recompute(t, seg, mb.sb[seg & 1]);
      if (!grid_sync(gb)) return;
    }
  }
  for (int seg = a.nseg - 1; seg >= 0; --seg) {
    const int t0 = seg * L, t1 = min(t0 + L, T);
    const int nb = t1 - t0, nr = seg > 0 ? L - 1 : 0;   // segment seg-1 is a full one
    const int n = nb > nr ? nb : nr;
    for (int i = 0; i < n; ++i) {
      if (i < nb) {
        const int t = t1 - 1 - i;
        if (t < Tf) adjoint(t, seg, mb.sb[seg & 1]);
      }
      if (i < nr) {
        const int t = (seg - 1) * L + i;
        if (t < Tf) recompute(t, seg - 1, mb.sb[(seg - 1) & 1]);
      }
      if (!grid_sync(gb)) return;
    }
    flush();
  }
  {   // dtheta += (d rinit / dtheta)^T adjoint(x^F_{-1}) (the output of step 0 has parity 1)
    const float* lx0 = mb.lx + ((size_t)1 * a.F + f) * DX * J;
    for (int j = j0; j < J; j += stride) {
      float z0[NZ0];
      own_normals<M, M::NZ0, INJ>(a, f, j, 0, z0);
      float l[DX];
#pragma unroll
      for (int d = 0; d < DX; ++d) l[d] = lx0[d * J + j];
      M::bwd_init(c, z0, l, gs);
      fold();
    }
    flush();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NG; i += TPB) {
    double sum = 0.0;
#pragma unroll 1
    for (int w = 0; w < NW; ++w) sum += s_g[w][i];
    mb.gpart[(size_t)blockIdx.x * kMaxNG + i] = sum;
  }
}

// The persistent adjoint with a split-phase barrier, for launches where every
// thread owns one particle j (CTAs x threads >= J).  The iterations are those
// of k_mop_bwd_persist in the same order (recompute of the last segment, then
// per segment the backward steps interleaved with the recomputation of the
// segment before), decoded from one flat index, so every float64 gradient sum
// is formed in the same order and the results are identical.  Between
// iterations a CTA arrives at the counting barrier right after its stores,
// then does the next iteration's work that reads nothing written by other
// CTAs in the current one -- the forward quantities of its backward step
// (state, normals, log-density, pi, first-child offsets) and its
// recomputation's ancestor and normals -- and only then waits.  What remains
// after the wait is the children's adjoint sums and the parent gather.
template <class M, int TPB, bool INJ>
__global__ void __launch_bounds__(TPB) k_mop_bwd_split(Args a, MopBwdP mb, GridBar gb) {
  constexpr int DX = M::MAXDX, NG = M::NG, NW = TPB / 32;
  constexpr int NZ = M::NZ > 0 ? M::NZ : 1, NZ0 = M::NZ0 > 0 ? M::NZ0 : 1;
  __shared__ typename M::Consts c;
  __shared__ double s_g[NW][NG];
  __shared__ int s_ok;
  const int f = blockIdx.x / mb.nbf, cb = blockIdx.x % mb.nbf;
  const int u = filter_unit(a, f), Tf = filter_len(a, u);
  const int J = a.J, T = a.T, L = a.ckpt_every, nseg = a.nseg;
  load_consts<M>(a, f, c);
  for (int i = threadIdx.x; i < NW * NG; i += TPB) (&s_g[0][0])[i] = 0.0;
  __syncthreads();
  const int j = cb * TPB + threadIdx.x;
  const bool act = j < J;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t sbf = (size_t)f * L * DX * J;
  const float* ckf = a.mop_ckpt + (size_t)f * nseg * DX * J;
  constexpr bool GD = NG <= 32;
  float gs[NG];
  double gd[GD ? NG : 1];
#pragma unroll
  for (int i = 0; i < NG; ++i) gs[i] = 0.0f;
#pragma unroll
  for (int i = 0; i < (GD ? NG : 1); ++i) gd[i] = 0.0;
  auto fold = [&]() {
    if (GD) {
#pragma unroll
      for (int i = 0; i < NG; ++i) {
        gd[i] += (double)gs[i];
        gs[i] = 0.0f;
      }
    }
  };
  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i < NG; ++i) {
      const double v = warp_sum_f64(GD ? gd[GD ? i : 0] : (double)gs[i]);
      if (lane == 0) s_g[warp][i] += v;
      gs[i] = 0.0f;
      if (GD) gd[GD ? i : 0] = 0.0;
    }
  };
  auto xin_of = [&](int t, int seg) -> const float* {
    const int t0 = seg * L;
    return (t == t0) ? ckf + (size_t)seg * DX * J : mb.sb[seg & 1] + sbf + (size_t)(t - 1 - t0) * DX * J;
  };
  // iteration q: backward step ta of segment sa (or -1), recomputation of
  // step tr of segment sr (or -1), and whether segment sa's sums are flushed
  const int nb_last = T - (nseg - 1) * L;
  const int n0 = nb_last > 1 ? nb_last - 1 : 0;
  const int n_last = max(nb_last, nseg > 1 ? L - 1 : 0);
  const int Q = n0 + n_last + (nseg - 1) * L;
  auto sched = [&](int q, int& ta, int& sa, int& tr, int& sr, bool& fl) {
    ta = -1; tr = -1; sa = 0; sr = 0; fl = false;
    if (q < n0) { tr = (nseg - 1) * L + q; sr = nseg - 1; return; }
    int qq = q - n0, seg, i, n;
    if (qq < n_last) { seg = nseg - 1; i = qq; n = n_last; }
    else { qq -= n_last; seg = nseg - 2 - qq / L; i = qq % L; n = L; }
    const int t0 = seg * L, t1 = min(t0 + L, T);
    const int nb = t1 - t0, nr = seg > 0 ? L - 1 : 0;
    if (i < nb) { ta = t1 - 1 - i; sa = seg; }
    if (i < nr) { tr = (seg - 1) * L + i; sr = seg - 1; }
    fl = (i == n - 1);
  };
  // work of iteration q that reads only the forward's saves and this
  // thread's own earlier writes
  float px[DX], pz[NZ], pm = 0.0f, ppi = 0.0f, rz[NZ];
  int plo = 0, phi = 0, rj = 0;
  typename M::Keep kp;
  auto prefetch = [&](int q) {
    int ta, sa, tr, sr;
    bool fl;
    sched(q, ta, sa, tr, sr, fl);
    if (act && ta >= 0 && ta < Tf) {
      const float* xin = xin_of(ta, sa);
#pragma unroll
      for (int d = 0; d < DX; ++d) px[d] = xin[(size_t)d * J + j];
      own_normals<M, M::NZ, INJ>(a, f, j, ta + 1, pz);
      Obs<M> ob;
      ob.load(a, u, ta);
      pm = M::fwd_keep(c, ob.y, ob.yc, px, pz, kp);
      const float Mt = a.mop_M[(size_t)f * T + ta];
      const double S1 = a.mop_S[(size_t)f * T + ta];
      ppi = 0.0f;
      if (S1 > 0.0 && pm == pm) ppi = (float)((double)pp_expf(pm - Mt) / S1);
      const int* off = a.mop_off + ((size_t)f * T + ta) * (J + 1);
      plo = off[j];
      phi = off[j + 1];
    }
    if (act && tr >= 0 && tr < Tf) {
      rj = a.anc[((size_t)f * T + tr) * J + j];
      own_normals<M, M::NZ, INJ>(a, f, rj, tr + 1, rz);
    }
  };
  auto wait = [&](unsigned int epoch) -> bool {
    if (threadIdx.x == 0) {
      int ok = 1;
      const unsigned int target = epoch * gb.n;
      long long i = 0;
      while ((int)(ld_acquire_u32(gb.count) - target) < 0) {
        if (++i > gb.cap || ld_relaxed_u32(gb.abort) != 0u) { ok = 0; break; }
        __nanosleep(20);
      }
      if (!ok) {
        atomicOr(gb.err, 1u);
        atomicExch(gb.abort, 1u);
      }
      s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
  };

  prefetch(0);
  for (int q = 0; q < Q; ++q) {
    if (q > 0 && !wait((unsigned)q)) return;
    int ta, sa, tr, sr;
    bool fl;
    sched(q, ta, sa, tr, sr, fl);
    if (act && ta >= 0 && ta < Tf) {
      const int pin = ta & 1, pout = pin ^ 1;
      const float* lxi = mb.lx + ((size_t)pin * a.F + f) * DX * J;
      const float* lwi = mb.lw + ((size_t)pin * a.F + f) * J;
      float lx[DX];
#pragma unroll
      for (int d = 0; d < DX; ++d) lx[d] = 0.0f;
      float lw = 0.0f;
      // a parent of many children (degenerate weights): several loads in flight,
      // the sums still taken in child order
#pragma unroll 4
      for (int k = plo; k < phi; ++k) {
#pragma unroll
        for (int d = 0; d < DX; ++d) lx[d] += lxi[(size_t)d * J + k];
        lw += lwi[k];
      }
      const float gl = -1.0f;
      const float lm = lw + gl * ppi;
      const float lwP = lw + gl * (ppi - 1.0f / (float)J);
      if (pm == pm && pm > -INFINITY) {
        add_process_weight<DX>(lx, a.pwi, lwP);
        M::bwd(c, px, pz, kp, lm, lx, gs);
        fold();
      } else {
#pragma unroll
        for (int d = 0; d < DX; ++d) lx[d] = 0.0f;
      }
      float* lxo = mb.lx + ((size_t)pout * a.F + f) * DX * J;
      float* lwo = mb.lw + ((size_t)pout * a.F + f) * J;
#pragma unroll
      for (int d = 0; d < DX; ++d) lxo[(size_t)d * J + j] = lx[d];
      lwo[j] = mb.alpha * lwP;
    }
    if (act && tr >= 0 && tr < Tf) {
      const float* xin = xin_of(tr, sr);
      float* xo = mb.sb[sr & 1] + sbf + (size_t)(tr - sr * L) * DX * J;
      float x[DX];
#pragma unroll
      for (int d = 0; d < DX; ++d) x[d] = xin[(size_t)d * J + rj];
      M::rproc(c, x, rz);
#pragma unroll
      for (int d = 0; d < DX; ++d) xo[(size_t)d * J + j] = x[d];
    }
    if (fl) flush();
    if (q + 1 < Q) {
      __syncthreads();   // every thread's stores before the arrival (release)
      if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(gb.count) : "memory");
      prefetch(q + 1);
    }
  }
  {   // dtheta += (d rinit / dtheta)^T adjoint(x^F_{-1}): this thread's own
      // adjoint of step 0 (parity 1), written above
    if (act) {
      const float* lx0 = mb.lx + ((size_t)1 * a.F + f) * DX * J;
      float z0[NZ0];
      own_normals<M, M::NZ0, INJ>(a, f, j, 0, z0);
      float l[DX];
#pragma unroll
      for (int d = 0; d < DX; ++d) l[d] = lx0[(size_t)d * J + j];
      M::bwd_init(c, z0, l, gs);
      fold();
    }
    flush();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NG; i += TPB) {
    double sum = 0.0;
#pragma unroll 1
    for (int w = 0; w < NW; ++w) sum += s_g[w][i];
    mb.gpart[(size_t)blockIdx.x * kMaxNG + i] = sum;
  }
}

// Natural-scale gradient sums of filter f (its CTAs' totals, in CTA order),
// chained to the estimation scale as k_mop_chain does.
template <class M>
__global__ void k_mop_chain_parts(Args a, const double* gpart, int nbf, double* grad) {
  __shared__ double gn[kMaxNG];
  const int f = blockIdx.x;
  for (int i = threadIdx.x; i < kMaxNG; i += blockDim.x) {
    double sum = 0.0;
    if (i < M::NG)
      for (int c = 0; c < nbf; ++c) sum += gpart[((size_t)f * nbf + c) * kMaxNG + i];
    gn[i] = sum;
  }
  __syncthreads();
  const int P = a.model.n_params;
  for (int p = threadIdx.x; p < P; p += blockDim.x)
    grad[(size_t)f * P + p] = Chain<M>::map(a.model, a.theta + (size_t)f * P, gn, p, (a.flags & PPF_F_EST) != 0);
}

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------

static int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      n = 0;
  }
  return n;
}

// CTAs of `kernel` that fit on the device at once (0 when unknown).
template <class K>
static int coresident(K kernel, int tpb, size_t smem) {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, tpb, smem) != cudaSuccess) return 0;
  return per * num_sms();
}

static GridBar grid_bar(const Args& a, unsigned int n) {
  GridBar g;
  g.count = a.gbar;
  g.gen = a.gbar + 1;
  g.abort = a.gbar + 2;
  g.err = a.err;
  g.n = n;
  g.cap = a.spin_cap;
  return g;
}

template <class K, class... Args_>
static int launch_coop(K kernel, int grid, int tpb, size_t smem, cudaStream_t s, Args_... args) {
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(tpb);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...) == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

// The persistent forward with TILE = TPB * IT particles per CTA; PPF_EUNSUPPORTED
// when the F * ntiles CTAs cannot all be resident at once.
template <class M, int TPB, int IT, bool INJ>
static int mop_forward_persist_t(Args& a, cudaStream_t s) {
  constexpr int TILE = TPB * IT;
  const size_t smem = sizeof(float) * M::MAXDX * TILE + sizeof(int) * (TILE + 4) + sizeof(float) * TILE;
  auto kern = k_mop_fwd_persist<M, TPB, IT, INJ>;
  const int ntiles = (a.J + TILE - 1) / TILE;
  const long long grid = (long long)a.F * ntiles;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return PPF_ECUDA;
  if (grid > coresident(kern, TPB, smem)) return PPF_EUNSUPPORTED;
  a.tile = TILE;
  a.ntiles = ntiles;
  k_prep<M><<<(a.F + 127) / 128, 128, 0, s>>>(a);
  PROF_BEGIN(KIND_MOP_FWD);
  const int rc = launch_coop(kern, (int)grid, TPB, smem, s, a, grid_bar(a, (unsigned)grid));
  PROF_END(KIND_MOP_FWD);
  return rc;
}

template <class M, bool INJ>
static int mop_backward_persist_t(Args& a, const MopWork& w, cudaStream_t s) {
  constexpr int TPB = 256;
  constexpr int DX = M::MAXDX;
  auto kern = k_mop_bwd_persist<M, TPB, INJ>;
  auto kern_split = k_mop_bwd_split<M, TPB, INJ>;
  const int want = (a.J + TPB - 1) / TPB;
  // one particle per thread: the split-phase form, when all its CTAs fit
  const bool split = (long long)a.F * want <= coresident(kern_split, TPB, 0);
  const int cap = split ? a.F * want : coresident(kern, TPB, 0);
  const int nbf = want < cap / a.F ? want : cap / a.F;
  if (nbf < 1 || !w.sb2 || !w.gpart) return PPF_EUNSUPPORTED;
  // the counting barrier's arrivals start from zero (with the generation and
  // abort words of the other form)
  if (cudaMemsetAsync(a.gbar, 0, 3 * sizeof(unsigned int), s) != cudaSuccess) return PPF_ECUDA;
  if (cudaMemsetAsync(w.lx, 0, sizeof(float) * 2ull * a.F * DX * a.J, s) != cudaSuccess) return PPF_ECUDA;
  if (cudaMemsetAsync(w.lw, 0, sizeof(float) * 2ull * a.F * a.J, s) != cudaSuccess) return PPF_ECUDA;
  MopBwdP mb;
  memset(&mb, 0, sizeof(mb));
  mb.sb[0] = w.sb;
  mb.sb[1] = w.sb2;
  mb.lx = w.lx;
  mb.lw = w.lw;
  mb.gpart = w.gpart;
  mb.alpha = w.alpha;
  mb.nbf = nbf;
  const int grid = a.F * nbf;
  PROF_BEGIN(KIND_MOP_BWD);
  int rc = split ? launch_coop(kern_split, grid, TPB, 0, s, a, mb, grid_bar(a, (unsigned)grid))
               : launch_coop(kern, grid, TPB, 0, s, a, mb, grid_bar(a, (unsigned)grid));
  PROF_END(KIND_MOP_BWD);
  if (rc) return rc;
  k_mop_chain_parts<M><<<a.F, 64, 0, s>>>(a, w.gpart, nbf, w.grad);
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

// The grid-resident forward: C CTAs of 512 threads per filter, as many as fit
// on the device at once (up to kGridMaxC per filter, at least 128 particles per
// CTA), each CTA's slice at most 2048 particles.  PPF_EUNSUPPORTED when the
// shape does not fit (the caller then takes the per-step kernels).
template <class M, bool INJ>
static int mop_forward_grid(Args& a, cudaStream_t s) {
  constexpr int TPB = 512;
  constexpr int kMaxJC = 2048;
  if (!a.slotw || (a.flags & (PPF_F_ESS | PPF_F_FMEAN | PPF_F_PMEAN))) return PPF_EUNSUPPORTED;
  auto kern = k_mop_fwd_grid<M, TPB, INJ>;
  auto smem_of = [](int jc) { return sizeof(float) * (M::MAXDX + 1) * jc + sizeof(int) * (jc + 4); };
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_of(kMaxJC)) !=
      cudaSuccess)
    return PPF_ECUDA;
  const int cap = coresident(kern, TPB, smem_of(kMaxJC));
  int C = cap / a.F;
  C = C < kGridMaxC ? C : kGridMaxC;
  const int cmax = (a.J + 127) / 128;
  C = C < cmax ? C : cmax;
  if (C < 1 || (long long)a.F * C > kMaxGridSlots) return PPF_EUNSUPPORTED;
  const int JC = (((a.J + C - 1) / C) + 3) & ~3;
  if (JC > kMaxJC) return PPF_EUNSUPPORTED;
  C = (a.J + JC - 1) / JC;
  const int grid = a.F * C;
  // the inboxes (tag 0: not yet written)
  if ((long long)grid * C > kInboxWords) return PPF_EUNSUPPORTED;
  if (cudaMemsetAsync(a.slotw, 0, sizeof(uint64_t) * 6 * (size_t)grid * C, s) != cudaSuccess) return PPF_ECUDA;
  k_prep<M><<<(a.F + 127) / 128, 128, 0, s>>>(a);
  PROF_BEGIN(KIND_MOP_FWD);
  const int rc = launch_coop(kern, grid, TPB, smem_of(JC), s, a, C, JC);
  PROF_END(KIND_MOP_FWD);
  return rc;
}

// Persistent launches apply to few filters: the forward's CTAs and the
// adjoint's must all fit on the device at once.  The grid-resident forward
// comes first; failing that, the tiled form with grid barriers takes
// 512-particle tiles when they need no more CTAs than there are SMs (one tile
// per SM: fewer barrier arrivals and tile totals to add per step), else
// 256-particle tiles.
template <class M, bool INJ>
static int mop_forward_persist(Args& a, cudaStream_t s) {
  {
    const int rc = mop_forward_grid<M, INJ>(a, s);
    if (rc != PPF_EUNSUPPORTED) return rc;
  }
  const long long t512 = (long long)a.F * ((a.J + 511) / 512);
  int rc = PPF_EUNSUPPORTED;
  if (t512 <= num_sms()) rc = mop_forward_persist_t<M, 128, 4, INJ>(a, s);
  if (rc != PPF_EUNSUPPORTED) return rc;
  rc = mop_forward_persist_t<M, 64, 4, INJ>(a, s);
  if (rc != PPF_EUNSUPPORTED) return rc;
  return mop_forward_persist_t<M, 128, 4, INJ>(a, s);
}

static bool want_persist(const Args& a) { return !(a.flags & PPF_F_NO_PERSIST) && a.gbar; }

template <class M, bool INJ>
int mop_backward(Args& a, const MopWork& w, cudaStream_t s) {
  constexpr int TPB = 256;
  constexpr int DX = M::MAXDX;
  const int J = a.J, T = a.T, L = a.ckpt_every;
  dim3 grid((J + TPB - 1) / TPB, a.F);
  if (cudaMemsetAsync(w.lx, 0, sizeof(float) * 2ull * a.F * DX * J, s) != cudaSuccess) return PPF_ECUDA;
  if (cudaMemsetAsync(w.lw, 0, sizeof(float) * 2ull * a.F * J, s) != cudaSuccess) return PPF_ECUDA;
  if (cudaMemsetAsync(w.gnat, 0, sizeof(double) * (size_t)a.F * kMaxNG, s) != cudaSuccess) return PPF_ECUDA;
  MopBwd mb;
  memset(&mb, 0, sizeof(mb));
  mb.gnat = w.gnat;
  mb.alpha = w.alpha;
  const size_t ck_fs = (size_t)a.nseg * DX * J;    // checkpoint filter stride
  const size_t sb_fs = (size_t)L * DX * J;         // segment-buffer filter stride
  for (int seg = a.nseg - 1; seg >= 0; --seg) {
    const int t0 = seg * L;
    const int t1 = (t0 + L < T) ? t0 + L : T;
    // recompute x^F_t, t in [t0, t1-1), into the segment buffer
    PROF_BEGIN(KIND_MOP_RECOMP);
    for (int t = t0; t < t1 - 1; ++t) {
      mb.xin = (t == t0) ? a.mop_ckpt + (size_t)seg * DX * J : w.sb + (size_t)(t - 1 - t0) * DX * J;
      mb.xin_fs = (t == t0) ? ck_fs : sb_fs;
      mb.xout = w.sb + (size_t)(t - t0) * DX * J;
      mb.xout_fs = sb_fs;
      k_mop_recomp<M, TPB, INJ><<<grid, TPB, 0, s>>>(a, mb, t);
    }
    PROF_END(KIND_MOP_RECOMP);
    PROF_BEGIN(KIND_MOP_BWD);
    for (int t = t1 - 1; t >= t0; --t) {
      mb.xin = (t == t0) ? a.mop_ckpt + (size_t)seg * DX * J : w.sb + (size_t)(t - 1 - t0) * DX * J;
      mb.xin_fs = (t == t0) ? ck_fs : sb_fs;
      const int pin = t & 1, pout = pin ^ 1;
      mb.lx_in = w.lx + (size_t)pin * a.F * DX * J;
      mb.lw_in = w.lw + (size_t)pin * a.F * J;
      mb.lx_out = w.lx + (size_t)pout * a.F * DX * J;
      mb.lw_out = w.lw + (size_t)pout * a.F * J;
      k_mop_bwd<M, TPB, INJ><<<grid, TPB, 0, s>>>(a, mb, t);
    }
    PROF_END(KIND_MOP_BWD);
  }
  mb.lx_in = w.lx + (size_t)1 * a.F * DX * J;      // adjoint of x^F_{-1} (output of step 0)
  k_mop_bwd_init<M, TPB, INJ><<<grid, TPB, 0, s>>>(a, mb);
  k_mop_chain<M><<<a.F, 64, 0, s>>>(a, w.gnat, w.grad);
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M>
int run_mop_backward_model(Args& a, const MopWork& w, cudaStream_t s) {
  const bool inj = (a.flags & PPF_F_INJECT) != 0;
  if constexpr (M::WIDE) {
    // the wide LG: per-step adjoint launches, Philox draws
    if (inj) return PPF_EUNSUPPORTED;
    return mop_backward<M, false>(a, w, s);
  } else {
    if (want_persist(a)) {
      const int rc = inj ? mop_backward_persist_t<M, true>(a, w, s) : mop_backward_persist_t<M, false>(a, w, s);
      if (rc != PPF_EUNSUPPORTED) return rc;
    }
    return inj ? mop_backward<M, true>(a, w, s) : mop_backward<M, false>(a, w, s);
  }
}

template <class M>
int run_mop_model(Args& a, const MopWork& w, cudaStream_t s) {
  const bool inj = (a.flags & PPF_F_INJECT) != 0;
  int rc = PPF_EUNSUPPORTED;
  if constexpr (!M::WIDE) {
    if (want_persist(a)) rc = inj ? mop_forward_persist<M, true>(a, s) : mop_forward_persist<M, false>(a, s);
  }
  if (rc == PPF_EUNSUPPORTED) rc = run_stream_any(a, s);
  if (rc || !w.grad) return rc;
  return run_mop_backward_model<M>(a, w, s);
}

int run_mop(Args& a, const MopWork& w, cudaStream_t s) {
  switch (a.model.kind) {
        case PPF_MODEL_LG:
      return with_lg<int>(a.model, true, PPF_EUNSUPPORTED,
                          [&](auto tg) { return run_mop_model<typename decltype(tg)::type>(a, w, s); });
    case PPF_MODEL_SV: return run_mop_model<SV>(a, w, s);
    case PPF_MODEL_RICKER: return run_mop_model<Ricker>(a, w, s);
    default: return PPF_EINVAL;
  }
}



int run_mop_backward(Args& a, const MopWork& w, cudaStream_t s) {
  switch (a.model.kind) {
        case PPF_MODEL_LG:
      return with_lg<int>(a.model, true, PPF_EUNSUPPORTED, [&](auto tg) {
        return run_mop_backward_model<typename decltype(tg)::type>(a, w, s);
      });
    case PPF_MODEL_SV: return run_mop_backward_model<SV>(a, w, s);
    case PPF_MODEL_RICKER: return run_mop_backward_model<Ricker>(a, w, s);
    default: return PPF_EINVAL;
  }
}

}  // namespace ppf
