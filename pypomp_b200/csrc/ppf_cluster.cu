// ppf_cluster.cu -- cluster-resident filters for small swarms.
//
// A filter whose swarm is too small to fill the GPU through the streaming
// kernels (few filters of a few thousand to ~10^5 particles: the IF2 unit
// filters of a panel, a single large-ish filter) is latency-bound there: every
// observation costs two dependent launches over a handful of CTAs.  Here one
// thread-block cluster of NC CTAs (NC <= 16, one per SM) owns one filter for
// the whole time loop.  CTA c keeps particles [c JC, (c+1) JC) -- state,
// log-weight and, for IF2, the parameter vector -- in its shared memory.
//
// CTAs exchange per-step numbers by PUSHING them: CTA c writes its numbers
// into slot c of every CTA's slot array (distributed shared memory stores,
// which need no round trip), and after the next cluster barrier each CTA
// reads all slots from its own shared memory.  Per observation:
//   A. every CTA finds the swarm's max / min / NaN key in its slots (pushed
//      by the producers of the weights at the end of the previous step), forms
//      its slice's fixed-point weights, block-scans them and pushes the slice
//      total; cluster barrier;
//   B. every CTA sums the slots (the exclusive prefix of its slice and the
//      filter total), computes the exact systematic first-child offsets of its
//      own parents (the same integer walk as the streaming path) and
//      propagates their children, writing each child's state and weight
//      straight into the shared memory of the CTA that owns the child's index;
//      it reduces the max / min / NaN of the weights it produced and pushes
//      them; cluster barrier.
// Two cluster barriers per observation.  The arithmetic is the streaming
// path's (same Philox streams per particle, same fixed-point CDF, same
// offsets), so results are bit-identical to it and to the oracle.  Cluster
// barriers are hardware barriers (barrier.cluster): no spin loop, and every
// CTA of a cluster runs the same number of them.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include <mutex>

#include "ppf.h"
#include "ppf_core.cuh"
#include "ppf_internal.h"
#include "ppf_kernels.cuh"
#include "ppf_models.cuh"

namespace cg = cooperative_groups;

namespace ppf {

constexpr int kClusterTPB = 512;
constexpr int kMaxCluster = 16;

// What CTA c publishes to the CTAs of its cluster: slot c of each CTA's array.
struct Slot {
  unsigned int maxkey, minkey, nan, pad;  // keys of the weights c produced for the next observation
  unsigned long long sum;                 // fixed-point weight sum of c's slice
  double s2, fx[4], px[4];                // ESS / mean sums of c's slice (pushed to CTA 0 only)
};

// What finalize_step reads of one step, kept by CTA 0 until the flush.
constexpr int kRecSteps = 32;
template <int DX>
struct StepRec {
  unsigned int maxkey, nan;
  double s2, fx[DX], px[DX];
  unsigned long long tot;
};

// Dynamic shared memory of one CTA, in 4-byte words: X[2][DX][JC], W[2][JC],
// (IF2) TH[2][P][JC], st[JC + 4], (IF2) per-thread parameter rows [TPB][P|1].
template <class M, bool IF2>
size_t cluster_smem_words(int JC, int P, int TPB) {
  size_t w = 2ull * M::MAXDX * JC + 2ull * JC + (size_t)JC + 4;
  if (IF2) w += 2ull * P * JC + (size_t)TPB * (P | 1);
  return w;
}

// Block max / min / NaN of the weights a CTA produced, pushed into slot c of
// every CTA of the cluster.  One barrier: warp reductions land in smk, then
// lanes 0..NC-1 of warp 0 each reduce all warps' values and push.  smk is
// written again only after the cluster barrier that follows.
template <int TPB>
__device__ __forceinline__ void push_maxmin(cg::cluster_group& cl, Slot* slots, int c, int NC,
                                            unsigned int mx, unsigned int mn, unsigned int nn,
                                            unsigned int* smk) {
  constexpr int NW = TPB / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  mx = warp_max_u32(mx);
  mn = warp_min_u32(mn);
  nn = __any_sync(0xffffffffu, nn != 0u) ? 1u : 0u;
  if (lane == 0) {
    smk[warp] = mx;
    smk[NW + warp] = mn;
    smk[2 * NW + warp] = nn;
  }
  __syncthreads();
  if ((int)threadIdx.x < NC) {
    unsigned int a = 0u, b = 0xffffffffu, o = 0u;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      a = max(a, smk[w]);
      b = min(b, smk[NW + w]);
      o |= smk[2 * NW + w];
    }
    Slot* dst = cl.map_shared_rank(slots, (int)threadIdx.x) + c;
    dst->maxkey = a;
    dst->minkey = b;
    dst->nan = o;
  }
}

template <class M, int TPB, bool IF2, bool INJ>
__global__ void __launch_bounds__(TPB, 1) k_cluster(Args a, int JC) {
  cg::cluster_group cl = cg::this_cluster();
  constexpr int DX = M::MAXDX;
  constexpr int G = ChildGroup<M::NZ>::G;
  extern __shared__ __align__(16) float smf[];
  __shared__ Slot slots[kMaxCluster];
  __shared__ typename M::Consts csh;
  __shared__ uint64_t s_scan[TPB / 32 + 1];
  __shared__ unsigned int smk[3 * (TPB / 32)];
  __shared__ double sd[TPB / 32];
  __shared__ StepRec<DX> s_rec[kRecSteps];     // CTA 0: the steps not yet added to the log-likelihood
  __shared__ double s_rll[kRecSteps];

  const int NC = (int)cl.num_blocks();
  const int c = (int)cl.block_rank();
  const int f = blockIdx.y;
  const int u = filter_unit(a, f);
  const int Tf = filter_len(a, u);
  const int J = a.J, P = a.model.n_params;
  const int base = c * JC;
  const int nc = max(0, min(JC, J - base));
  const bool est = (a.flags & PPF_F_EST) != 0;
  float* X[2];
  float* W[2];
  float* TH[2] = {nullptr, nullptr};
  X[0] = smf;
  X[1] = X[0] + DX * JC;
  W[0] = X[1] + DX * JC;
  W[1] = W[0] + JC;
  float* rest = W[1] + JC;
  if (IF2) {
    TH[0] = rest;
    TH[1] = TH[0] + P * JC;
    rest = TH[1] + P * JC;
  }
  int* st = reinterpret_cast<int*>(rest);
  float* th = IF2 ? reinterpret_cast<float*>(st + JC + 4) + threadIdx.x * if2_row_stride(P) : nullptr;
  const float log1e18 = pp_logf(1e-18f);
  const bool want_ess = (a.flags & PPF_F_ESS) != 0, want_fm = (a.flags & PPF_F_FMEAN) != 0;
  const bool want_pm = (a.flags & PPF_F_PMEAN) != 0;
  const bool want_sums = want_ess || want_fm || want_pm;

  if (!IF2 && threadIdx.x == 0) M::prepare(csh, a.theta + (size_t)f * P, a.model, est);
  __syncthreads();

  // ---- initial states, propagated into observation 0 -----------------------
  {
    Obs<M> ob;
    ob.load(a, u, 0);
    float* logw0 = a.logw ? a.logw + (size_t)f * a.T * J : nullptr;
    unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
    for (int l = threadIdx.x; l < nc; l += TPB) {
      const int k = base + l;
      float x[DX];
      float m;
      if (IF2) {
        for (int p = 0; p < P; ++p) th[p] = a.swarm_in[((size_t)f * P + p) * J + k];
        perturb_row<INJ>(a, f, k, 0, P, a.cool0[u], a.rw_sig0, th);
        typename M::Consts ci;
        M::prepare(ci, th, a.model, est);
        float z0[M::NZ0 > 0 ? M::NZ0 : 1];
        step_noise<M>(a, f, k, 0, M::NZ0, z0);
        M::rinit(ci, z0, x);
        perturb_row<INJ>(a, f, k, 1, P, a.cool[(size_t)u * a.T], a.rw_sig, th);
        M::prepare(ci, th, a.model, est);
        float z[M::NZ];
        step_noise<M>(a, f, k, 1, M::NZ, z);
        m = if2_measure(step1<M>(ci, ob, x, z), log1e18);
        for (int p = 0; p < P; ++p) TH[0][p * JC + l] = th[p];
      } else {
        const typename M::Consts cr = csh;
        float z0[M::NZ0 > 0 ? M::NZ0 : 1];
        step_noise<M>(a, f, k, 0, M::NZ0, z0);
        M::rinit(cr, z0, x);
        float z[M::NZ];
        step_noise<M>(a, f, k, 1, M::NZ, z);
        m = step1<M>(cr, ob, x, z);
      }
      const float w = a.base_init + m;
#pragma unroll
      for (int d = 0; d < DX; ++d) X[0][d * JC + l] = x[d];
      W[0][l] = w;
      accum_maxmin(w, mx, mn, nn);
      if (logw0) logw0[k] = w;
    }
    push_maxmin<TPB>(cl, slots, c, NC, mx, mn, nn, smk);
  }
  cl.sync();

  // the filter's log-likelihood, kept by thread 0 of CTA 0 and written once at
  // the end rather than read and written in global memory every observation
  double ll_acc = 0.0;
  const int ITC = (JC + TPB - 1) / TPB;        // parents per thread (contiguous)
  const int l0 = threadIdx.x * ITC;
  const int l1 = min(l0 + ITC, nc);
  for (int t = 0; t < Tf; ++t) {
    const int pc = t & 1, pn = pc ^ 1;
    const bool last = (t == Tf - 1);
    const float* Wc = W[pc];
    // the next observation, fetched now so its latency hides behind phase A
    Obs<M> ob;
    if (!last) ob.load(a, u, t + 1);
    const float coolt = (IF2 && !last) ? a.cool[(size_t)u * a.T + t + 1] : 0.0f;

    // A. max / min / NaN of the swarm from every producer's slot
    Acc acc;
    acc.maxkey = 0u;
    acc.minkey = 0xffffffffu;
    acc.nan = 0u;
    acc.pad = 0u;
    acc.s2 = 0.0;
    for (int d = 0; d < M::MAXDX; ++d) { acc.fx[d] = 0.0; acc.px[d] = 0.0; }   // the model's dimensions only
    for (int r = 0; r < NC; ++r) {
      acc.maxkey = max(acc.maxkey, slots[r].maxkey);
      acc.minkey = min(acc.minkey, slots[r].minkey);
      acc.nan |= slots[r].nan;
    }
    const bool nanf = acc.nan != 0;
    const float Mx = keyf(acc.maxkey);
    const bool collapsed = !nanf && Mx == -INFINITY;
    const bool qc = nanf || Mx == -INFINITY;

    // fixed-point weights of the slice: totals and this thread's prefix
    uint64_t qs = 0;
    double s2 = 0.0, fx[DX], px[DX];
    // the first QC fixed-point weights stay in registers for the offsets below
    constexpr int QC = 4;
    uint64_t qk[QC];
#pragma unroll
    for (int d = 0; d < DX; ++d) { fx[d] = 0.0; px[d] = 0.0; }
    for (int l = l0; l < l1; ++l) {
      const uint64_t q = qweight(Wc[l], Mx, qc);
#pragma unroll
      for (int i = 0; i < QC; ++i)
        if (l - l0 == i) qk[i] = q;
      qs += q;
      if (want_sums) {
        const double e = qc ? 1.0 : (double)pp_expf(Wc[l] - Mx);
        s2 += e * e;
#pragma unroll
        for (int d = 0; d < DX; ++d) {
          const double xv = (double)X[pc][d * JC + l];
          fx[d] += xv * e;
          px[d] += xv;
        }
      }
    }
    uint64_t btot;
    const uint64_t tex = block_excl_scan_u64_1b<TPB>(qs, s_scan, btot);
    if (want_sums) {
      Slot* o0 = cl.map_shared_rank(slots, 0) + c;
      const double b2 = block_sum_f64<TPB>(s2, sd);
      if (threadIdx.x == 0) o0->s2 = b2;
#pragma unroll
      for (int d = 0; d < DX; ++d) {
        const double bf = block_sum_f64<TPB>(fx[d], sd);
        const double bp = block_sum_f64<TPB>(px[d], sd);
        if (threadIdx.x == 0) { o0->fx[d] = bf; o0->px[d] = bp; }
      }
    }
    if ((int)threadIdx.x < NC) (cl.map_shared_rank(slots, (int)threadIdx.x) + c)->sum = btot;
    cl.sync();

    // B. filter total, this slice's prefix, the step's log-likelihood
    uint64_t E = 0, tot = 0;
    for (int r = 0; r < NC; ++r) {
      const uint64_t v = slots[r].sum;
      E += (r < c) ? v : 0ull;
      tot += v;
    }
    if (c == 0 && threadIdx.x == 0) {
      if (want_sums)
        for (int r = 0; r < NC; ++r) {
          acc.s2 += slots[r].s2;
          for (int d = 0; d < DX; ++d) { acc.fx[d] += slots[r].fx[d]; acc.px[d] += slots[r].px[d]; }
        }
      // the step's log-likelihood term is formed later (flush below): its
      // float64 log would otherwise hold CTA 0, and so the cluster, every step
      StepRec<DX>& rec = s_rec[t % kRecSteps];
      rec.maxkey = acc.maxkey;
      rec.nan = acc.nan;
      rec.s2 = acc.s2;
      for (int d = 0; d < DX; ++d) { rec.fx[d] = acc.fx[d]; rec.px[d] = acc.px[d]; }
      rec.tot = tot;
    }
    const bool rs = decide_resample(a, acc);

    // first-child offsets of this CTA's parents (global child indices)
    float lt32 = 0.0f;
    if (rs) {
      const Offsets o = make_offsets(tot, resample_u32(a, f, t), J);
      if (l0 < nc) {
        uint64_t C = E + tex;
        OffWalk wk = offwalk_init(o, C);
        st[l0] = wk.k;
        for (int l = l0; l < l1; ++l) {
          uint64_t q = 0;
#pragma unroll
          for (int i = 0; i < QC; ++i)
            if (l - l0 == i) q = qk[i];
          if (l - l0 >= QC) q = qweight(Wc[l], Mx, qc);
          const int kn = offwalk_add_c(o, wk, C, q);
          if (l + 1 < l1 || l + 1 == nc) st[l + 1] = kn;
        }
      }
    } else {
      if (nanf) lt32 = __int_as_float(0x7fc00000);
      else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
      for (int l = l0; l < l1; ++l) st[l] = base + l;
      if (l0 < nc && l1 == nc) st[nc] = base + nc;
    }
    __syncthreads();

    // children of this CTA's parents, into the owners' shared memory
    unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
    if (nc > 0) {
      const int klo = st[0], khi = st[nc];
      const float nwc = -pp_logf((float)J);
      int* anc = a.anc ? a.anc + ((size_t)f * a.T + t) * J : nullptr;
      float* logw = (a.logw && !last) ? a.logw + ((size_t)f * a.T + t + 1) * J : nullptr;
      const typename M::Consts cr = csh;
      // one child k of parent l with its process normals z
      auto child = [&](int k, int l, const float* z) {
        if (anc) anc[k] = base + l;
        if (last) {
          if (IF2)
            for (int p = 0; p < P; ++p) a.swarm_out[((size_t)f * P + p) * J + k] = TH[pc][p * JC + l];
          return;
        }
        float x[DX];
#pragma unroll
        for (int d = 0; d < DX; ++d) x[d] = X[pc][d * JC + l];
        float m;
        if (IF2) {
          for (int p = 0; p < P; ++p) th[p] = TH[pc][p * JC + l];
          perturb_row<INJ>(a, f, k, t + 2, P, coolt, a.rw_sig, th);
          typename M::Consts cc;
          M::prepare(cc, th, a.model, est);
          m = if2_measure(step1<M>(cc, ob, x, z), log1e18);
        } else {
          m = step1<M>(cr, ob, x, z);
        }
        const float wb = rs ? a.base_rs : (collapsed ? nwc : Wc[l] - lt32);
        const float w = wb + m;
        accum_maxmin(w, mx, mn, nn);
        const int r = k / JC, lk = k - r * JC;
        float* xr = cl.map_shared_rank(X[pn], r);
#pragma unroll
        for (int d = 0; d < DX; ++d) xr[d * JC + lk] = x[d];
        cl.map_shared_rank(W[pn], r)[lk] = w;
        if (IF2) {
          float* tr = cl.map_shared_rank(TH[pn], r);
          for (int p = 0; p < P; ++p) tr[p * JC + lk] = th[p];
        }
        if (logw) logw[k] = w;
      };
      if (khi - klo <= 2 * TPB) {
        // the usual case, about one child per parent: one child per thread
        // at a time, so every thread works and the step's critical path is
        // one child long; each thread draws its own child's normals (the
        // same numbers as the grouped draw below)
#pragma unroll 1
        for (int k = klo + (int)threadIdx.x; k < khi; k += TPB) {
          float z[M::NZ];
          if (!last) step_noise<M>(a, f, k, t + 2, M::NZ, z);
          child(k, find_parent(st, nc, k), z);
        }
      } else {
        // many children (a few heavy parents): groups of G consecutive
        // children per thread share their Philox blocks
        const int kA = klo & ~3;
        const int ngr = (khi - kA + G - 1) / G;
        const int g0 = (int)(((long long)threadIdx.x * ngr) / TPB);
        const int g1 = (int)(((long long)(threadIdx.x + 1) * ngr) / TPB);
        if (g0 < g1) {
          int l = find_parent(st, nc, max(kA + G * g0, klo));
#pragma unroll 1
          for (int g = g0; g < g1; ++g) {
            const int k0 = kA + G * g;
            if (k0 >= khi) break;
            float z[G * M::NZ];
            if (!last) group_noise_g<G, M::NZ, INJ>(a, f, t + 2, k0, z);
#pragma unroll
            for (int e = 0; e < G; ++e) {
              const int k = k0 + e;
              if (k < klo || k >= khi) continue;
              int adv = 0;
              while (l + 1 < nc && st[l + 1] <= k) {
                ++l;
                if (++adv > 8) { l = find_parent(st, nc, k); break; }
              }
              child(k, l, z + e * M::NZ);
            }
          }
        }
      }
    }
    if (!last) push_maxmin<TPB>(cl, slots, c, NC, mx, mn, nn, smk);
    cl.sync();   // children and slots visible to their owners; nobody leaves while others write to it
    // every kRecSteps steps (and after the last) CTA 0 forms the buffered
    // steps' terms in parallel and adds them in step order, as one thread
    // adding each step's term in turn would
    if (c == 0 && ((t + 1) % kRecSteps == 0 || t == Tf - 1)) {
      const int n = t % kRecSteps + 1, tb = t + 1 - n;
      __syncthreads();
      if ((int)threadIdx.x < n) {
        const StepRec<DX>& rec = s_rec[threadIdx.x];
        Acc ra;
        ra.maxkey = rec.maxkey;
        ra.minkey = rec.maxkey;
        ra.nan = rec.nan;
        ra.pad = 0u;
        ra.s2 = rec.s2;
        for (int d = 0; d < DX; ++d) { ra.fx[d] = rec.fx[d]; ra.px[d] = rec.px[d]; }
        double v = 0.0;
        finalize_step(a, f, tb + (int)threadIdx.x, ra, rec.tot, &v);
        s_rll[threadIdx.x] = v;
      }
      __syncthreads();
      if (threadIdx.x == 0)
        for (int i = 0; i < n; ++i) ll_acc += s_rll[i];
    }
  }
  if (c == 0 && threadIdx.x == 0) a.loglik[f] = ll_acc;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// Launch attributes: the largest dynamic shared memory any plan asks for and,
// for 16-CTA clusters, the non-portable cluster size.
template <class M, bool IF2, bool INJ>
static bool cluster_attrs() {
  auto kern = k_cluster<M, kClusterTPB, IF2, INJ>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kResidentSmemMax) != cudaSuccess ||
      cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return true;
}

static cudaLaunchConfig_t cluster_config(int NC, int F, size_t smem, cudaStream_t s, cudaLaunchAttribute* at) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(NC, F, 1);
  cfg.blockDim = dim3(kClusterTPB, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = NC;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

// How many clusters of NC CTAs with `smem` bytes each can be resident at once
// (cudaOccupancyMaxActiveClusters), cached per kernel, cluster size and size
// class of the shared memory; 0 when the query fails.
struct OccEntry {
  const void* fn;
  int nc, smem_kb, n;
};
static OccEntry g_occ[64];
static int g_occ_n = 0;
static std::mutex g_occ_mu;

template <class M, bool IF2, bool INJ>
static int max_active_clusters(int NC, size_t smem) {
  auto kern = k_cluster<M, kClusterTPB, IF2, INJ>;
  const void* fn = reinterpret_cast<const void*>(kern);
  const int kb = (int)((smem + 4095) / 4096) * 4;
  {
    std::lock_guard<std::mutex> lk(g_occ_mu);
    for (int i = 0; i < g_occ_n; ++i)
      if (g_occ[i].fn == fn && g_occ[i].nc == NC && g_occ[i].smem_kb == kb) return g_occ[i].n;
  }
  int n = 0;
  if (cluster_attrs<M, IF2, INJ>()) {
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = cluster_config(NC, 1, (size_t)kb * 1024, nullptr, at);
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
  }
  std::lock_guard<std::mutex> lk(g_occ_mu);
  if (g_occ_n < 64) g_occ[g_occ_n++] = OccEntry{fn, NC, kb, n};
  return n;
}

// Cluster size and slice: the largest cluster (<= 16 CTAs) that keeps at least
// 256 particles per CTA (2 CTAs at the least) and fits the slice in one CTA's
// shared memory.  With one_wave, also all F filters' clusters resident at once
// (the automatic choice: a second wave would double the time).
template <class M, bool IF2, bool INJ>
static bool cluster_plan_t(const Args& a, bool one_wave, int& NC, int& JC) {
  for (int n = kMaxCluster; n >= 2; n >>= 1) {
    const int jc = ((a.J + n - 1) / n + 3) & ~3;
    if (jc < 256 && n != 2) continue;
    const size_t smem = cluster_smem_words<M, IF2>(jc, a.model.n_params, kClusterTPB) * 4;
    if (smem > (size_t)kResidentSmemMax) continue;
    if (one_wave && max_active_clusters<M, IF2, INJ>(n, smem) < a.F) continue;
    NC = n;
    JC = jc;
    return true;
  }
  return false;
}

template <class M, bool IF2, bool INJ>
static int run_cluster_t(Args& a, cudaStream_t s) {
  int NC = 0, JC = 0;
  if (!cluster_plan_t<M, IF2, INJ>(a, true, NC, JC) && !cluster_plan_t<M, IF2, INJ>(a, false, NC, JC))
    return PPF_EUNSUPPORTED;
  if (max_active_clusters<M, IF2, INJ>(NC, cluster_smem_words<M, IF2>(JC, a.model.n_params, kClusterTPB) * 4) < 1)
    return PPF_EUNSUPPORTED;
  const size_t smem = cluster_smem_words<M, IF2>(JC, a.model.n_params, kClusterTPB) * 4;
  if (!cluster_attrs<M, IF2, INJ>()) return PPF_ECUDA;
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = cluster_config(NC, a.F, smem, s, at);
  PROF_BEGIN(KIND_CLUSTER);
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k_cluster<M, kClusterTPB, IF2, INJ>, a, JC);
  PROF_END(KIND_CLUSTER);
  return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M, bool IF2>
static int run_cluster_m(Args& a, cudaStream_t s) {
  return (a.flags & PPF_F_INJECT) ? run_cluster_t<M, IF2, true>(a, s) : run_cluster_t<M, IF2, false>(a, s);
}

template <class M, bool IF2>
static bool fits_m(const Args& a) {
  int NC = 0, JC = 0;
  return (a.flags & PPF_F_INJECT) ? cluster_plan_t<M, IF2, true>(a, true, NC, JC)
                                  : cluster_plan_t<M, IF2, false>(a, true, NC, JC);
}

template <bool IF2>
static bool fits_any(const Args& a) {
  switch (a.model.kind) {
        case PPF_MODEL_LG:
      return with_lg<bool>(a.model, false, false,
                           [&](auto tg) { return fits_m<typename decltype(tg)::type, IF2>(a); });
    case PPF_MODEL_SV: return fits_m<SV, IF2>(a);
    case PPF_MODEL_RICKER: return fits_m<Ricker, IF2>(a);
    default: return false;
  }
}

template <bool IF2>
static int run_any(Args& a, cudaStream_t s) {
  switch (a.model.kind) {
        case PPF_MODEL_LG:
      return with_lg<int>(a.model, false, PPF_EUNSUPPORTED,
                          [&](auto tg) { return run_cluster_m<typename decltype(tg)::type, IF2>(a, s); });
    case PPF_MODEL_SV: return run_cluster_m<SV, IF2>(a, s);
    case PPF_MODEL_RICKER: return run_cluster_m<Ricker, IF2>(a, s);
    default: return PPF_EINVAL;
  }
}

// True when the automatic choice may use the cluster path: a plan exists with
// all filters resident in one wave.
bool cluster_fits(const Args& a, bool if2) {
  if (a.mode == MODE_MOP) return false;
  return if2 ? fits_any<true>(a) : fits_any<false>(a);
}

int run_cluster(Args& a, bool if2, cudaStream_t s) {
  if (a.mode == MODE_MOP) return PPF_EUNSUPPORTED;
  return if2 ? run_any<true>(a, s) : run_any<false>(a, s);
}

}  // namespace ppf
