// ppf_pfilter.cu -- the batched bootstrap particle filter on sm_100a.
//
// Replaces the per-observation loop of pypomp's _pfilter_internal /
// _pfilter_step (pypomp/core/algorithms/pfilter.py:15-182), with
// _normalize_weights (helpers.py:34-57), _resample (helpers.py:14-31) and
// _resampler (helpers.py:60-91).  Three execution paths share one arithmetic
// definition (ppf.h) and so produce bit-identical results:
//
//  STREAM   (large J): particle state in HBM, structure of arrays
//           X[F][dx][J], W[F][J], two kernels per observation:
//             k_sum      fixed-point weights, block sums, single-pass
//                        decoupled-lookback prefix over the tiles of a filter
//             k_resprop  tile CDF, closed-form systematic offsets per parent,
//                        child expansion by a max-scan in shared memory, and
//                        the NEXT step's rproc + dmeas fused for each child
//                        (the gather reads the parent from shared memory).
//  RESIDENT (small J): one CTA per filter holds the swarm in shared memory for
//           the whole time loop: one launch per call.
//  PLAIN    (1x baseline): one filter at a time, four textbook kernels per
//           step (propagate, block scan, scan of block sums, binary-search
//           ancestors) with ancestors and CDF in global memory.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <algorithm>
#include <vector>

#include "ppf.h"
#include "ppf_core.cuh"
#include "ppf_models.cuh"
#include "ppf_internal.h"

namespace ppf {

// ------------------------------ shared helpers ------------------------------

template <class M>
__device__ __forceinline__ void step_noise(const Args& a, int f, int j, int s, int n, float* z) {
  if (a.flags & PPF_F_INJECT) {
    if (s == 0) {
      for (int i = 0; i < n; ++i) z[i] = a.inj_z0[((size_t)f * a.J + j) * n + i];
    } else {
      const size_t base = (((size_t)f * a.T + (s - 1)) * a.J + j) * n;
      for (int i = 0; i < n; ++i) z[i] = a.inj_z[base + i];
    }
  } else {
    pp_normals(a.seeds[f], (uint32_t)j, (uint32_t)s, PPF_TAG_PROCESS, n, z);
  }
}

__device__ __forceinline__ uint32_t resample_u32(const Args& a, int f, int t) {
  if (a.flags & PPF_F_INJECT) return pp_u32_from_float(a.inj_u[(size_t)f * a.T + t]);
  return pp_resample_u32(a.seeds[f], (uint32_t)(t + 1));
}

__device__ __forceinline__ int filter_len(const Args& a, int u) { return a.T_u ? a.T_u[u] : a.T; }
__device__ __forceinline__ int filter_unit(const Args& a, int f) { return a.unit ? a.unit[f] : 0; }

// rproc into observation t (step s = t+1) and dmeas at observation t.
template <class M>
__device__ __forceinline__ float propagate(const Args& a, const typename M::Consts& c, int f, int u,
                                           int j, int t, float* x) {
  float z[M::MAXDX > 0 ? M::MAXDX : 1];
  const int nz = M::n_step(c);
  step_noise<M>(a, f, j, t + 1, nz, z);
  M::rproc(c, x, z);
  const float* y = a.ys + ((size_t)u * a.T + t) * a.model.dy;
  const float yc = a.ycon ? a.ycon[(size_t)u * a.T + t] : 0.0f;
  return M::dmeas(c, y, yc, x);
}

// Finalise one observation of one filter: log-likelihood term and outputs.
__device__ void finalize_step(const Args& a, int f, int t, const Acc& acc, uint64_t tot, double* loglik) {
  const bool nanf = acc.nan != 0;
  const float Mx = keyf(acc.maxkey);
  const bool collapsed = !nanf && Mx == -INFINITY;
  double ll;
  if (nanf) ll = __longlong_as_double(0x7ff8000000000000ll);
  else if (collapsed) ll = -INFINITY;
  else ll = (double)Mx + log((double)tot) - 40.0 * kLn2 - (a.mode == MODE_MOP ? log((double)a.J) : 0.0);
  *loglik += ll;
  if ((a.flags & PPF_F_CLL) && a.cll) a.cll[(size_t)f * a.T + t] = ll;
  const double S1 = (double)tot * 9.094947017729282e-13;  // 2^-40
  if ((a.flags & PPF_F_ESS) && a.ess) {
    float e;
    if (nanf) e = __int_as_float(0x7fc00000);
    else if (collapsed) e = (float)a.J;
    else e = (float)(S1 * S1 / acc.s2);
    a.ess[(size_t)f * a.T + t] = e;
  }
  const int dx = a.model.dx;
  if ((a.flags & PPF_F_FMEAN) && a.fmean)
    for (int d = 0; d < dx; ++d)
      a.fmean[((size_t)f * a.T + t) * dx + d] = (float)(collapsed ? acc.px[d] / a.J : acc.fx[d] / S1);
  if ((a.flags & PPF_F_PMEAN) && a.pmean)
    for (int d = 0; d < dx; ++d) a.pmean[((size_t)f * a.T + t) * dx + d] = (float)(acc.px[d] / a.J);
}

__device__ __forceinline__ bool decide_resample(const Args& a, const Acc& acc) {
  if (acc.nan) return false;
  const float Mx = keyf(acc.maxkey);
  if (Mx == -INFINITY) return 0.0f > a.logthresh;
  const float mn = keyf(acc.minkey);
  return (Mx - mn) > a.logthresh;
}

__device__ __forceinline__ void accum_maxmin(float w, unsigned int& mx, unsigned int& mn, unsigned int& nn) {
  if (w != w || w == INFINITY) { nn = 1u; return; }
  const unsigned int k = fkey(w);
  mx = max(mx, k);
  mn = min(mn, k);
}

// ============================================================================
// STREAM path
// ============================================================================

template <class M, int TPB>
__global__ void __launch_bounds__(TPB) k_init(Args a) {
  __shared__ typename M::Consts c;
  __shared__ unsigned int smk[2 * (TPB / 32)];
  __shared__ double sd[TPB / 32];
  const int f = blockIdx.y;
  const int u = filter_unit(a, f);
  if (threadIdx.x == 0) M::prepare(c, a.theta + (size_t)f * a.model.n_params, a.model, (a.flags & PPF_F_EST) != 0);
  __syncthreads();
  const int dx = a.model.dx;
  float* X = a.X[0] + (size_t)f * dx * a.J;
  float* W = a.W[0] + (size_t)f * a.J;
  unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
  double px[M::MAXDX];
  for (int d = 0; d < M::MAXDX; ++d) px[d] = 0.0;
  const int j0 = blockIdx.x * a.tile;
  const int j1 = min(j0 + a.tile, a.J);
  for (int j = j0 + threadIdx.x; j < j1; j += TPB) {
    float z[M::MAXDX > 0 ? M::MAXDX : 1];
    float x[M::MAXDX];
    step_noise<M>(a, f, j, 0, M::n_init(c), z);
    M::rinit(c, z, x);
    const float m = propagate<M>(a, c, f, u, j, 0, x);
    const float w = (a.mode == MODE_MOP ? 0.0f : a.base_init) + m;
    for (int d = 0; d < dx; ++d) { X[(size_t)d * a.J + j] = x[d]; px[d] += (double)x[d]; }
    W[j] = w;
    if (a.logw) a.logw[((size_t)f * a.T) * a.J + j] = w;
    accum_maxmin(w, mx, mn, nn);
  }
  block_maxmin_u32<TPB>(mx, mn, smk);
  nn = __syncthreads_or(nn);
  Acc* acc = a.acc[0] + f;
  if (threadIdx.x == 0) {
    atomicMax(&acc->maxkey, mx);
    atomicMin(&acc->minkey, mn);
    if (nn) atomicOr(&acc->nan, 1u);
    if (blockIdx.x == 0) a.loglik[f] = 0.0;
  }
  if (a.flags & PPF_F_PMEAN) {
    for (int d = 0; d < dx; ++d) {
      const double s = block_sum_f64<TPB>(px[d], sd);
      if (threadIdx.x == 0) atomicAdd(&acc->px[d], s);
    }
  }
}

// Fixed-point sums of the weights of one tile, then the decoupled-lookback
// prefix over the tiles of the filter (Merrill & Garland 2016).
template <class M, int TPB, int IT>
__global__ void __launch_bounds__(TPB) k_sum(Args a, int t) {
  constexpr int TILE = TPB * IT;
  __shared__ int s_v;
  __shared__ uint64_t s_scan[TPB / 32 + 1];
  __shared__ double sd[TPB / 32];
  __shared__ uint64_t s_excl;
  if (threadIdx.x == 0) s_v = atomicAdd(a.counter + (t & 1), 1);
  __syncthreads();
  const int v = s_v;
  if (v >= a.ntiles * a.F) {  // defensive: a stale counter must not index past the batch
    if (threadIdx.x == 0) atomicOr(a.err, 4u);
    return;
  }
  const int f = v / a.ntiles, b = v % a.ntiles;
  const int u = filter_unit(a, f);
  if (t >= filter_len(a, u)) return;
  const int p = t & 1;
  const Acc acc = a.acc[p][f];
  if (b == 0 && threadIdx.x == 0) {
    Acc* nx = a.acc[p ^ 1] + f;
    nx->maxkey = 0u; nx->minkey = 0xffffffffu; nx->nan = 0u;
    nx->s2 = 0.0;
    for (int d = 0; d < 4; ++d) { nx->fx[d] = 0.0; nx->px[d] = 0.0; }
  }
  const bool nanf = acc.nan != 0;
  const float Mx = keyf(acc.maxkey);
  const bool collapsed = nanf || Mx == -INFINITY;
  const float* W = a.W[p] + (size_t)f * a.J;
  const int jb = b * TILE + threadIdx.x * IT;
  uint64_t qs = 0;
  double s2 = 0.0;
  float wv[IT];
#pragma unroll
  for (int i = 0; i < IT; ++i) wv[i] = (jb + i < a.J) ? W[jb + i] : -INFINITY;
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    if (jb + i < a.J) {
      const uint64_t q = qweight(wv[i], Mx, collapsed);
      qs += q;
      if (a.flags & PPF_F_ESS) {
        const double e = collapsed ? 1.0 : (double)pp_expf(wv[i] - Mx);
        s2 += e * e;
      }
    }
  }
  uint64_t btot;
  block_excl_scan_u64<TPB>(qs, s_scan, btot);
  uint64_t* desc = a.desc[p] + (size_t)f * a.ntiles;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    uint64_t excl = 0;
    if (b == 0) {
      if (lane == 0) st_release_u64(desc, kStatusIncl | btot);
    } else {
      if (lane == 0) st_release_u64(desc + b, kStatusAgg | btot);
      int pos = b - 1;
      long long spins = 0;
      bool timed_out = false;
      while (true) {
        const int idx = pos - lane;
        uint64_t d = idx >= 0 ? ld_acquire_u64(desc + idx) : kStatusIncl;
        while (__any_sync(0xffffffffu, (d >> 62) == 0ull)) {
          if (++spins > kSpinCap) { timed_out = true; break; }
          if ((d >> 62) == 0ull) { __nanosleep(32); d = ld_acquire_u64(desc + idx); }
        }
        if (timed_out) break;
        const unsigned int inc = __ballot_sync(0xffffffffu, (d >> 62) == 2ull);
        if (inc) {
          const int first = __ffs(inc) - 1;
          excl += warp_sum_u64(lane <= first ? (d & kValueMask) : 0ull);
          break;
        }
        excl += warp_sum_u64(d & kValueMask);
        pos -= 32;
      }
      if (timed_out && lane == 0) atomicOr(a.err, 1u);
      if (lane == 0) st_release_u64(desc + b, kStatusIncl | (excl + btot));
    }
    if (lane == 0) {
      s_excl = excl;
      a.excl[(size_t)f * a.ntiles + b] = excl;
      if (b == a.ntiles - 1) a.tot[f] = excl + btot;
    }
  }
  if (a.flags & PPF_F_ESS) {
    const double s = block_sum_f64<TPB>(s2, sd);
    if (threadIdx.x == 0) atomicAdd(&a.acc[p][f].s2, s);
  }
  if (a.flags & PPF_F_FMEAN) {
    const float* X = a.X[p] + (size_t)f * a.model.dx * a.J;
    for (int d = 0; d < a.model.dx; ++d) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < IT; ++i)
        if (jb + i < a.J) {
          const double e = collapsed ? 1.0 : (double)pp_expf(wv[i] - Mx);
          s += (double)X[(size_t)d * a.J + jb + i] * e;
        }
      s = block_sum_f64<TPB>(s, sd);
      if (threadIdx.x == 0) atomicAdd(&a.acc[p][f].fx[d], s);
    }
  }
}

// Resample the parents of one tile and propagate their children to the next
// observation (rproc + dmeas fused), writing the next step's X, W.
template <class M, int TPB, int IT>
__global__ void __launch_bounds__(TPB) k_resprop(Args a, int t) {
  constexpr int TILE = TPB * IT;
  constexpr int CH = TILE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* xs = reinterpret_cast<float*>(smem_raw);                       // [dx][TILE]
  int* mk = reinterpret_cast<int*>(smem_raw + sizeof(float) * M::MAXDX * TILE);  // [CH]
  __shared__ typename M::Consts c;
  __shared__ uint64_t s_scan[TPB / 32 + 1];
  __shared__ int s_mx[TPB / 32 + 1];
  __shared__ unsigned int smk[2 * (TPB / 32)];
  __shared__ double sd[TPB / 32];
  __shared__ int s_klo, s_khi;

  const int f = blockIdx.y, b = blockIdx.x;
  const int u = filter_unit(a, f);
  const int Tf = filter_len(a, u);
  const int p = t & 1;
  // reset the next step's lookback descriptors and tile counter (before any
  // early exit: finished filters of a ragged panel still own these slots)
  if (threadIdx.x == 0) {
    a.desc[p ^ 1][(size_t)f * a.ntiles + b] = 0ull;
    if (b == 0 && f == 0) a.counter[p ^ 1] = 0;
  }
  if (t >= Tf) return;
  const Acc acc = a.acc[p][f];
  const uint64_t tot = a.tot[f];
  if (b == 0 && threadIdx.x == 0) finalize_step(a, f, t, acc, tot, a.loglik + f);
  if (t == Tf - 1 && !(a.flags & PPF_F_SAVE_ANC)) return;
  if (threadIdx.x == 0) M::prepare(c, a.theta + (size_t)f * a.model.n_params, a.model, (a.flags & PPF_F_EST) != 0);
  const bool nanf = acc.nan != 0;
  const float Mx = keyf(acc.maxkey);
  const bool collapsed = !nanf && Mx == -INFINITY;
  const bool rs = decide_resample(a, acc);
  const int dx = a.model.dx;
  const float* Xc = a.X[p] + (size_t)f * dx * a.J;
  const float* Wc = a.W[p] + (size_t)f * a.J;
  float* Xn = a.X[p ^ 1] + (size_t)f * dx * a.J;
  float* Wn = a.W[p ^ 1] + (size_t)f * a.J;
  const bool last = (t == Tf - 1);
  unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
  double px[M::MAXDX];
  for (int d = 0; d < M::MAXDX; ++d) px[d] = 0.0;
  const float base = (a.mode == MODE_MOP) ? 0.0f : a.base_rs;
  const int jt = b * TILE;
  const int ntile = min(TILE, a.J - jt);
  __syncthreads();

  if (!rs) {
    // No resampling: every particle is its own child; weights carry over.
    float lt32 = 0.0f;
    if (nanf) lt32 = __int_as_float(0x7fc00000);
    else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
    for (int l = threadIdx.x; l < ntile; l += TPB) {
      const int j = jt + l;
      if (a.anc) a.anc[((size_t)f * a.T + t) * a.J + j] = j;
      if (last) continue;
      float x[M::MAXDX];
      for (int d = 0; d < dx; ++d) x[d] = Xc[(size_t)d * a.J + j];
      const float nw = collapsed ? -pp_logf((float)a.J) : Wc[j] - lt32;
      const float m = propagate<M>(a, c, f, u, j, t + 1, x);
      const float w = nw + m;
      for (int d = 0; d < dx; ++d) { Xn[(size_t)d * a.J + j] = x[d]; px[d] += (double)x[d]; }
      Wn[j] = w;
      if (a.logw) a.logw[((size_t)f * a.T + t + 1) * a.J + j] = w;
      accum_maxmin(w, mx, mn, nn);
    }
  } else {
    const uint32_t u32 = resample_u32(a, f, t);
    const uint64_t E = a.excl[(size_t)f * a.ntiles + b];
    // 1. fixed-point weights and their tile-local exclusive scan
    const int l0 = threadIdx.x * IT;
    uint64_t q[IT];
    uint64_t qs = 0;
#pragma unroll
    for (int i = 0; i < IT; ++i) {
      q[i] = (l0 + i < ntile) ? qweight(Wc[jt + l0 + i], Mx, collapsed) : 0ull;
      qs += q[i];
    }
    uint64_t btot;
    const uint64_t tex = block_excl_scan_u64<TPB>(qs, s_scan, btot);
    // 2. closed-form first-child offsets of each parent; stage parent states
    int st[IT], en[IT];
    {
      uint64_t C = E + tex;
      int prev = nchild(C, tot, u32, a.J);
      if (threadIdx.x == 0) s_klo = prev;
#pragma unroll
      for (int i = 0; i < IT; ++i) {
        C += q[i];
        const int e = (l0 + i < ntile) ? nchild(C, tot, u32, a.J) : prev;
        st[i] = prev; en[i] = e; prev = e;
      }
      if (l0 < ntile && l0 + IT >= ntile) s_khi = prev;
      if (ntile <= 0 && threadIdx.x == 0) s_khi = s_klo;
    }
    for (int l = threadIdx.x; l < ntile; l += TPB)
      for (int d = 0; d < dx; ++d) xs[d * TILE + l] = Xc[(size_t)d * a.J + jt + l];
    __syncthreads();
    const int klo = s_klo, khi = s_khi;
    // 3. expand children window by window: mark each parent's first child,
    //    max-scan the marks, then process the children in order.
    int carry = -1;
    for (int w0 = klo; w0 < khi; w0 += CH) {
      const int wn = min(CH, khi - w0);
      for (int i = threadIdx.x; i < CH; i += TPB) mk[i] = -1;
      __syncthreads();
#pragma unroll
      for (int i = 0; i < IT; ++i)
        if (en[i] > st[i] && st[i] >= w0 && st[i] < w0 + CH) mk[st[i] - w0] = l0 + i;
      __syncthreads();
      {
        constexpr int PER = CH / TPB;
        int loc[PER];
        int run = -1;
#pragma unroll
        for (int i = 0; i < PER; ++i) { run = max(run, mk[threadIdx.x * PER + i]); loc[i] = run; }
        int tmax;
        const int ex = block_excl_max_i32<TPB>(run, s_mx, tmax);
        const int base_c = max(ex, carry);
#pragma unroll
        for (int i = 0; i < PER; ++i) mk[threadIdx.x * PER + i] = max(base_c, loc[i]);
        carry = max(carry, tmax);
      }
      __syncthreads();
      for (int i = threadIdx.x; i < wn; i += TPB) {
        const int l = mk[i];
        const int k = w0 + i;
        if (l < 0 || l >= ntile) { atomicOr(a.err, 2u); continue; }  // defensive: never index out of the tile
        if (a.anc) a.anc[((size_t)f * a.T + t) * a.J + k] = jt + l;
        if (last) continue;
        float x[M::MAXDX];
        for (int d = 0; d < dx; ++d) x[d] = xs[d * TILE + l];
        const float m = propagate<M>(a, c, f, u, k, t + 1, x);
        const float w = base + m;
        for (int d = 0; d < dx; ++d) { Xn[(size_t)d * a.J + k] = x[d]; px[d] += (double)x[d]; }
        Wn[k] = w;
        if (a.logw) a.logw[((size_t)f * a.T + t + 1) * a.J + k] = w;
        accum_maxmin(w, mx, mn, nn);
      }
      __syncthreads();
    }
  }
  if (last) return;
  block_maxmin_u32<TPB>(mx, mn, smk);
  nn = __syncthreads_or(nn);
  Acc* an = a.acc[p ^ 1] + f;
  if (threadIdx.x == 0) {
    if (mx) atomicMax(&an->maxkey, mx);
    if (mn != 0xffffffffu) atomicMin(&an->minkey, mn);
    if (nn) atomicOr(&an->nan, 1u);
  }
  if (a.flags & PPF_F_PMEAN) {
    for (int d = 0; d < dx; ++d) {
      const double s = block_sum_f64<TPB>(px[d], sd);
      if (threadIdx.x == 0) atomicAdd(&an->px[d], s);
    }
  }
}

// ============================================================================
// RESIDENT path: one CTA per filter, the whole time loop in one launch.
// Shared memory: xs[dx][J] float, ws[J] float, mk[J] int.
// ============================================================================

template <class M, int TPB, int MAXIT>
__global__ void __launch_bounds__(TPB, 1) k_resident(Args a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int J = a.J;
  const int dx = a.model.dx;
  float* xs = reinterpret_cast<float*>(smem_raw);
  float* ws = xs + (size_t)dx * J;
  int* mk = reinterpret_cast<int*>(ws + J);
  __shared__ typename M::Consts c;
  __shared__ uint64_t s_scan[TPB / 32 + 1];
  __shared__ int s_mx[TPB / 32 + 1];
  __shared__ unsigned int smk[2 * (TPB / 32)];
  __shared__ double sd[TPB / 32];
  __shared__ Acc s_acc;
  __shared__ uint64_t s_tot;
  __shared__ double s_ll;

  const int f = blockIdx.x;
  const int u = filter_unit(a, f);
  const int Tf = filter_len(a, u);
  if (threadIdx.x == 0) {
    M::prepare(c, a.theta + (size_t)f * a.model.n_params, a.model, (a.flags & PPF_F_EST) != 0);
    s_ll = 0.0;
  }
  __syncthreads();
  // blocked ownership for the scan: thread owns [l0, l0+per)
  const int per = (J + TPB - 1) / TPB;
  const int l0 = min(J, threadIdx.x * per);
  const int l1 = min(J, l0 + per);

  // step 0: rinit + rproc + dmeas for every particle
  for (int j = threadIdx.x; j < J; j += TPB) {
    float z[M::MAXDX > 0 ? M::MAXDX : 1];
    float x[M::MAXDX];
    step_noise<M>(a, f, j, 0, M::n_init(c), z);
    M::rinit(c, z, x);
    const float m = propagate<M>(a, c, f, u, j, 0, x);
    const float w = (a.mode == MODE_MOP ? 0.0f : a.base_init) + m;
    for (int d = 0; d < dx; ++d) xs[d * J + j] = x[d];
    ws[j] = w;
    if (a.logw) a.logw[((size_t)f * a.T) * J + j] = w;
  }
  __syncthreads();
  const float base = (a.mode == MODE_MOP) ? 0.0f : a.base_rs;

  for (int t = 0; t < Tf; ++t) {
    // (a) max / min / nan and prediction-mean sums
    unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
    for (int j = l0; j < l1; ++j) accum_maxmin(ws[j], mx, mn, nn);
    block_maxmin_u32<TPB>(mx, mn, smk);
    nn = __syncthreads_or(nn);
    if (threadIdx.x == 0) {
      s_acc.maxkey = mx; s_acc.minkey = mn; s_acc.nan = nn; s_acc.s2 = 0.0;
      for (int d = 0; d < 4; ++d) { s_acc.fx[d] = 0.0; s_acc.px[d] = 0.0; }
    }
    __syncthreads();
    const bool nanf = s_acc.nan != 0;
    const float Mx = keyf(s_acc.maxkey);
    const bool collapsed = !nanf && Mx == -INFINITY;
    const bool qcollapsed = nanf || Mx == -INFINITY;
    // (b) fixed-point weights, scan, total
    uint64_t qs = 0;
    double s2 = 0.0;
    for (int j = l0; j < l1; ++j) {
      qs += qweight(ws[j], Mx, qcollapsed);
      if (a.flags & (PPF_F_ESS)) {
        const double e = qcollapsed ? 1.0 : (double)pp_expf(ws[j] - Mx);
        s2 += e * e;
      }
    }
    uint64_t tot;
    const uint64_t tex = block_excl_scan_u64<TPB>(qs, s_scan, tot);
    if (a.flags & PPF_F_ESS) {
      const double s = block_sum_f64<TPB>(s2, sd);
      if (threadIdx.x == 0) s_acc.s2 = s;
    }
    if (a.flags & (PPF_F_FMEAN | PPF_F_PMEAN)) {
      for (int d = 0; d < dx; ++d) {
        double sf = 0.0, sp = 0.0;
        for (int j = l0; j < l1; ++j) {
          const double xv = (double)xs[d * J + j];
          sp += xv;
          sf += xv * (qcollapsed ? 1.0 : (double)pp_expf(ws[j] - Mx));
        }
        sf = block_sum_f64<TPB>(sf, sd);
        sp = block_sum_f64<TPB>(sp, sd);
        if (threadIdx.x == 0) { s_acc.fx[d] = sf; s_acc.px[d] = sp; }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_tot = tot;
      double ll = s_ll;
      finalize_step(a, f, t, s_acc, tot, &ll);
      s_ll = ll;
    }
    __syncthreads();
    const bool last = (t == Tf - 1);
    if (last && !a.anc) break;
    const bool rs = decide_resample(a, s_acc);
    if (!rs) {
      float lt32 = 0.0f;
      if (nanf) lt32 = __int_as_float(0x7fc00000);
      else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
      if (a.anc)
        for (int j = threadIdx.x; j < J; j += TPB) a.anc[((size_t)f * a.T + t) * J + j] = j;
      if (last) break;
      for (int j = threadIdx.x; j < J; j += TPB) {
        float x[M::MAXDX];
        for (int d = 0; d < dx; ++d) x[d] = xs[d * J + j];
        const float nw = collapsed ? -pp_logf((float)J) : ws[j] - lt32;
        const float m = propagate<M>(a, c, f, u, j, t + 1, x);
        const float w = nw + m;
        for (int d = 0; d < dx; ++d) xs[d * J + j] = x[d];
        ws[j] = w;
        if (a.logw) a.logw[((size_t)f * a.T + t + 1) * J + j] = w;
      }
      __syncthreads();
      continue;
    }
    // (c) offsets and marks
    const uint32_t u32 = resample_u32(a, f, t);
    for (int j = threadIdx.x; j < J; j += TPB) mk[j] = -1;
    __syncthreads();
    {
      uint64_t C = tex;
      int prev = nchild(C, tot, u32, J);
      for (int j = l0; j < l1; ++j) {
        C += qweight(ws[j], Mx, qcollapsed);
        const int e = nchild(C, tot, u32, J);
        if (e > prev) mk[prev] = j;
        prev = e;
      }
    }
    __syncthreads();
    {
      int run = -1;
      for (int j = l0; j < l1; ++j) { run = max(run, mk[j]); mk[j] = run; }
      int tmax;
      const int ex = block_excl_max_i32<TPB>(run, s_mx, tmax);
      for (int j = l0; j < l1; ++j) mk[j] = max(mk[j], ex);
    }
    __syncthreads();
    if (a.anc)
      for (int k = threadIdx.x; k < J; k += TPB) a.anc[((size_t)f * a.T + t) * J + k] = mk[k];
    if (last) break;
    // (d) children: gather parent from shared memory, propagate, then store
    float nx[MAXIT][M::MAXDX];
    float nw[MAXIT];
#pragma unroll
    for (int it = 0; it < MAXIT; ++it) {
      const int k = threadIdx.x + it * TPB;
      if (k < J) {
        float x[M::MAXDX];
        int l = mk[k];
        if (l < 0 || l >= J) { atomicOr(a.err, 2u); l = 0; }  // defensive: never index outside the swarm
        for (int d = 0; d < dx; ++d) x[d] = xs[d * J + l];
        const float m = propagate<M>(a, c, f, u, k, t + 1, x);
#pragma unroll
        for (int d = 0; d < M::MAXDX; ++d) nx[it][d] = x[d];
        nw[it] = base + m;
      }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < MAXIT; ++it) {
      const int k = threadIdx.x + it * TPB;
      if (k < J) {
        for (int d = 0; d < dx; ++d) xs[d * J + k] = nx[it][d];
        ws[k] = nw[it];
        if (a.logw) a.logw[((size_t)f * a.T + t + 1) * J + k] = nw[it];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) a.loglik[f] = s_ll;
}

// ============================================================================
// PLAIN path: one filter per launch sequence.  Accumulators double-buffered
// by step parity (a.acc[p][0]); the no-resampling carry flag stays on device.
// ============================================================================

__device__ __forceinline__ void reset_acc(Acc* acc) {
  acc->maxkey = 0u; acc->minkey = 0xffffffffu; acc->nan = 0u; acc->s2 = 0.0;
  for (int d = 0; d < 4; ++d) { acc->fx[d] = 0.0; acc->px[d] = 0.0; }
}
__global__ void k_reset_acc(Acc* acc) { reset_acc(acc); }

template <class M, int TPB>
__global__ void __launch_bounds__(TPB) kp_prop(Args a, int f, int t) {
  __shared__ typename M::Consts c;
  __shared__ unsigned int smk[2 * (TPB / 32)];
  __shared__ double sd[TPB / 32];
  const int u = filter_unit(a, f);
  if (t >= filter_len(a, u)) return;
  if (threadIdx.x == 0) M::prepare(c, a.theta + (size_t)f * a.model.n_params, a.model, (a.flags & PPF_F_EST) != 0);
  __syncthreads();
  const int dx = a.model.dx;
  const int j = blockIdx.x * TPB + threadIdx.x;
  const int p = t & 1;
  unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
  double px[M::MAXDX];
  for (int d = 0; d < M::MAXDX; ++d) px[d] = 0.0;
  if (j < a.J) {
    float x[M::MAXDX];
    float w0;
    if (t == 0) {
      float z[M::MAXDX > 0 ? M::MAXDX : 1];
      step_noise<M>(a, f, j, 0, M::n_init(c), z);
      M::rinit(c, z, x);
      w0 = (a.mode == MODE_MOP ? 0.0f : a.base_init);
    } else {
      const int par = a.pl_anc[j];
      for (int d = 0; d < dx; ++d) x[d] = a.X[p ^ 1][(size_t)d * a.J + par];
      w0 = a.pl_carry_dev[0] ? a.W[p ^ 1][j] : (a.mode == MODE_MOP ? 0.0f : a.base_rs);
    }
    const float m = propagate<M>(a, c, f, u, j, t, x);
    const float w = w0 + m;
    for (int d = 0; d < dx; ++d) { a.X[p][(size_t)d * a.J + j] = x[d]; px[d] += (double)x[d]; }
    a.W[p][j] = w;
    if (a.logw) a.logw[((size_t)f * a.T + t) * a.J + j] = w;
    accum_maxmin(w, mx, mn, nn);
  }
  block_maxmin_u32<TPB>(mx, mn, smk);
  nn = __syncthreads_or(nn);
  Acc* acc = a.acc[p];
  if (threadIdx.x == 0) {
    if (t == 0 && blockIdx.x == 0) a.loglik[f] = 0.0;
    atomicMax(&acc->maxkey, mx);
    atomicMin(&acc->minkey, mn);
    if (nn) atomicOr(&acc->nan, 1u);
  }
  if (a.flags & PPF_F_PMEAN)
    for (int d = 0; d < dx; ++d) {
      const double s = block_sum_f64<TPB>(px[d], sd);
      if (threadIdx.x == 0) atomicAdd(&acc->px[d], s);
    }
}

template <int TPB>
__global__ void __launch_bounds__(TPB) kp_scan1(Args a, int f, int t) {
  __shared__ uint64_t s_scan[TPB / 32 + 1];
  __shared__ double sd[TPB / 32];
  if (t >= filter_len(a, filter_unit(a, f))) return;
  const int p = t & 1;
  const Acc acc = *a.acc[p];
  const float Mx = keyf(acc.maxkey);
  const bool qc = acc.nan != 0 || Mx == -INFINITY;
  const int j = blockIdx.x * TPB + threadIdx.x;
  const float w = j < a.J ? a.W[p][j] : 0.0f;
  const uint64_t q = j < a.J ? qweight(w, Mx, qc) : 0ull;
  uint64_t bt;
  const uint64_t ex = block_excl_scan_u64<TPB>(q, s_scan, bt);
  if (j < a.J) a.pl_cdf[j] = ex + q;
  if (threadIdx.x == 0) a.pl_bsum[blockIdx.x] = bt;
  if (a.flags & PPF_F_ESS) {
    const double e = (j < a.J) ? (qc ? 1.0 : (double)pp_expf(w - Mx)) : 0.0;
    const double s = block_sum_f64<TPB>(e * e, sd);
    if (threadIdx.x == 0) atomicAdd(&a.acc[p]->s2, s);
  }
  if (a.flags & PPF_F_FMEAN)
    for (int d = 0; d < a.model.dx; ++d) {
      const double e = (j < a.J) ? (qc ? 1.0 : (double)pp_expf(w - Mx)) * (double)a.X[p][(size_t)d * a.J + j] : 0.0;
      const double s = block_sum_f64<TPB>(e, sd);
      if (threadIdx.x == 0) atomicAdd(&a.acc[p]->fx[d], s);
    }
}

// single block: scan of the block sums, finalise the observation, and reset
// the accumulators of the next step.
template <int TPB>
__global__ void __launch_bounds__(TPB) kp_scan2(Args a, int f, int t, int nblk) {
  __shared__ uint64_t s_scan[TPB / 32 + 1];
  if (t >= filter_len(a, filter_unit(a, f))) return;
  const int p = t & 1;
  uint64_t carry = 0;
  for (int b0 = 0; b0 < nblk; b0 += TPB) {
    const int i = b0 + threadIdx.x;
    const uint64_t v = i < nblk ? a.pl_bsum[i] : 0ull;
    uint64_t bt;
    const uint64_t ex = block_excl_scan_u64<TPB>(v, s_scan, bt);
    if (i < nblk) a.pl_boff[i] = carry + ex;
    carry += bt;
  }
  if (threadIdx.x == 0) {
    a.tot[0] = carry;
    finalize_step(a, f, t, *a.acc[p], carry, a.loglik + f);
    reset_acc(a.acc[p ^ 1]);
  }
}

template <int TPB>
__global__ void __launch_bounds__(TPB) kp_anc(Args a, int f, int t) {
  if (t >= filter_len(a, filter_unit(a, f))) return;
  const int p = t & 1;
  const Acc acc = *a.acc[p];
  const uint64_t tot = a.tot[0];
  const int k = blockIdx.x * TPB + threadIdx.x;
  const bool rs = decide_resample(a, acc);
  if (k < a.J) {
    int par;
    if (rs) {
      const uint32_t u32 = resample_u32(a, f, t);
      const u128 R = ((u128)u32 + ((u128)k << 32)) * (u128)tot;
      const uint64_t Jsh = (uint64_t)a.J << 32;
      int lo = 0, hi = a.J;  // first j with C_j * J * 2^32 > R
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const uint64_t Cm = a.pl_cdf[mid] + a.pl_boff[mid / TPB];
        if ((u128)Cm * (u128)Jsh <= R) lo = mid + 1;
        else hi = mid;
      }
      par = lo;
    } else {
      par = k;
      const bool nanf = acc.nan != 0;
      const float Mx = keyf(acc.maxkey);
      float nw;
      if (nanf) nw = __int_as_float(0x7fc00000);
      else if (Mx == -INFINITY) nw = -pp_logf((float)a.J);
      else nw = a.W[p][k] - (Mx + pp_logf((float)tot * 9.094947017729282e-13f));
      a.W[p][k] = nw;
    }
    a.pl_anc[k] = par;
    if (a.anc) a.anc[((size_t)f * a.T + t) * a.J + k] = par;
  }
  if (k == 0) a.pl_carry_dev[0] = rs ? 0 : 1;
}

// ============================================================================
// Host dispatch
// ============================================================================

// Optional per-kernel timing (ppf_profile_begin / ppf_profile_end): CUDA
// events recorded on the launch stream around each kernel of the next calls.
Profiler g_prof;

void Profiler::mark(int kind, cudaStream_t s, bool start) {
  if (!enabled) return;
  if (start) {
    if (used >= (int)evs.size()) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      evs.push_back({a, b, 0});
    }
    evs[used].kind = kind;
    cudaEventRecord(evs[used].a, s);
  } else {
    cudaEventRecord(evs[used].b, s);
    ++used;
  }
}

#define PROF_BEGIN(kind) g_prof.mark(kind, s, true)
#define PROF_END(kind) g_prof.mark(kind, s, false)

template <class M>
int run_stream(Args& a, cudaStream_t s) {
  constexpr int TPB = 256, IT = 8, TILE = TPB * IT;
  a.tile = TILE;
  a.ntiles = (a.J + TILE - 1) / TILE;
  const size_t smem = sizeof(float) * M::MAXDX * TILE + sizeof(int) * TILE;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_resprop<M, TPB, IT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr_set = true;
  }
  dim3 grid(a.ntiles, a.F);
  PROF_BEGIN(KIND_INIT);
  k_init<M, TPB><<<grid, TPB, 0, s>>>(a);
  PROF_END(KIND_INIT);
  for (int t = 0; t < a.T; ++t) {
    PROF_BEGIN(KIND_SUM);
    k_sum<M, TPB, IT><<<a.ntiles * a.F, TPB, 0, s>>>(a, t);
    PROF_END(KIND_SUM);
    PROF_BEGIN(KIND_RESPROP);
    k_resprop<M, TPB, IT><<<grid, TPB, smem, s>>>(a, t);
    PROF_END(KIND_RESPROP);
  }
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M>
size_t resident_smem(const Args& a) {
  return (size_t)a.J * sizeof(float) * (a.model.dx + 1) + (size_t)a.J * sizeof(int);
}

template <class M, int MAXIT>
int launch_resident(Args& a, size_t smem, cudaStream_t s) {
  constexpr int TPB = 512;
  cudaFuncSetAttribute(k_resident<M, TPB, MAXIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  PROF_BEGIN(KIND_RESIDENT);
  k_resident<M, TPB, MAXIT><<<a.F, TPB, smem, s>>>(a);
  PROF_END(KIND_RESIDENT);
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M>
int run_resident(Args& a, cudaStream_t s) {
  constexpr int TPB = 512;
  const size_t smem = resident_smem<M>(a);
  const int per = (a.J + TPB - 1) / TPB;
  if (smem > kResidentSmemMax || per > 32) return PPF_EUNSUPPORTED;
  if (per <= 2) return launch_resident<M, 2>(a, smem, s);
  if (per <= 8) return launch_resident<M, 8>(a, smem, s);
  return launch_resident<M, 32>(a, smem, s);
}

template <class M>
int run_plain(Args& a, cudaStream_t s) {
  constexpr int TPB = 256;
  const int nblk = (a.J + TPB - 1) / TPB;
  for (int f = 0; f < a.F; ++f) {
    k_reset_acc<<<1, 1, 0, s>>>(a.acc[0]);
    for (int t = 0; t < a.T; ++t) {
      PROF_BEGIN(KIND_PLAIN);
      kp_prop<M, TPB><<<nblk, TPB, 0, s>>>(a, f, t);
      kp_scan1<TPB><<<nblk, TPB, 0, s>>>(a, f, t);
      kp_scan2<1024><<<1, 1024, 0, s>>>(a, f, t, nblk);
      kp_anc<TPB><<<nblk, TPB, 0, s>>>(a, f, t);
      PROF_END(KIND_PLAIN);
    }
  }
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

__global__ void k_reset_accs(Acc* acc, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) reset_acc(acc + i);
}

int reset_accumulators(Args& a, cudaStream_t s) {
  for (int i = 0; i < 2; ++i) k_reset_accs<<<(a.F + 127) / 128, 128, 0, s>>>(a.acc[i], a.F);
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M>
int dispatch_model(Args& a, int path, cudaStream_t s) {
  switch (path) {
    case PPF_PATH_PLAIN: return run_plain<M>(a, s);
    case PPF_PATH_STREAM: return run_stream<M>(a, s);
    case PPF_PATH_RESIDENT: return run_resident<M>(a, s);
    default: return PPF_EINVAL;
  }
}

int run_pfilter_path(Args& a, int path, cudaStream_t s) {
  switch (a.model.kind) {
    case PPF_MODEL_LG: return dispatch_model<LG>(a, path, s);
    case PPF_MODEL_SV: return dispatch_model<SV>(a, path, s);
    case PPF_MODEL_RICKER: return dispatch_model<Ricker>(a, path, s);
    default: return PPF_EINVAL;
  }
}

size_t resident_smem_bytes(const Args& a) {
  return (size_t)a.J * sizeof(float) * (a.model.dx + 1) + (size_t)a.J * sizeof(int);
}

}  // namespace ppf
