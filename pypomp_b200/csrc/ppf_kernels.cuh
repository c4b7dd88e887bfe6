// ppf_kernels.cuh -- device helpers shared by the particle-filter kernels
// (ppf_pfilter.cu) and the MOP kernels (ppf_mop.cu): noise, observations,
// per-step finalisation, the exact systematic-offset walk, constants.
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "ppf.h"
#include "ppf_core.cuh"
#include "ppf_internal.h"
#include "ppf_models.cuh"

namespace ppf {

// ------------------------------ shared helpers ------------------------------

__device__ __forceinline__ int filter_len(const Args& a, int u) { return a.T_u ? a.T_u[u] : a.T; }
__device__ __forceinline__ int filter_unit(const Args& a, int f) { return a.unit ? a.unit[f] : 0; }

// Normals of one particle (used by the plain path and by single particles).
template <class M>
__device__ __forceinline__ void step_noise(const Args& a, int f, int j, int s, int n, float* z) {
  if (n <= 0) return;
  if (a.flags & PPF_F_INJECT) {
    if (s == 0) {
      for (int i = 0; i < n; ++i) z[i] = a.inj_z0[((size_t)f * a.J + j) * n + i];
    } else {
      const size_t base = (((size_t)f * a.T + (s - 1)) * a.J + j) * n;
      for (int i = 0; i < n; ++i) z[i] = a.inj_z[base + i];
    }
  } else {
    pp_normals_own(a.seeds[f], (uint32_t)j, (uint32_t)s, PPF_TAG_PROCESS, n, z);
  }
}

// Normals of the group of 4 consecutive particles k0..k0+3 (k0 % 4 == 0) at
// step s, N per particle: z[e*N + r].  Philox calls (k0 N)/4 ... + N-1 cover
// the group exactly; positions past J read zeros in injection mode.
template <int N, bool INJ, bool FAST = false>
__device__ __forceinline__ void group_noise(const Args& a, int f, int s, int k0, float* z) {
  if (N == 0) return;
  if (INJ) {
    const float* src = (s == 0) ? a.inj_z0 + (size_t)f * a.J * N
                                : a.inj_z + (((size_t)f * a.T + (s - 1)) * a.J) * N;
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
      for (int r = 0; r < N; ++r) z[e * N + r] = (k0 + e < a.J) ? src[(size_t)(k0 + e) * N + r] : 0.0f;
  } else {
    const uint64_t seed = a.seeds[f];
    const uint32_t c0 = (uint32_t)(k0 / 4) * N;
#pragma unroll
    for (int c = 0; c < N; ++c) {
      if (FAST) pp_normal4_fast(seed, c0 + c, (uint32_t)s, PPF_TAG_PROCESS, z + 4 * c);
      else pp_normal4(seed, c0 + c, (uint32_t)s, PPF_TAG_PROCESS, z + 4 * c);
    }
  }
}

// Children per Philox group: a run of consecutive particles whose normals fill
// whole Philox blocks (G * NZ a multiple of 4), so every word is used.  Four
// children (two or more independent Philox chains for NZ >= 2) measured faster
// than the smallest group for the 2-D LG batch, the chains overlapping, and
// pairs of 4-D LG children spilled more than groups of four.
template <int NZ>
struct ChildGroup {
  static constexpr int G = 4;
  static_assert((G * NZ) % 4 == 0 || NZ == 0, "a group must fill whole Philox blocks");
};

// Normals of the G consecutive particles k0..k0+G-1 (k0 % G == 0) at step s,
// N per particle: z[e*N + r].  Philox calls (k0 N)/4 ... cover them exactly.
template <int G, int N, bool INJ, bool FAST = false>
__device__ __forceinline__ void group_noise_g(const Args& a, int f, int s, int k0, float* z) {
  if (N == 0) return;
  if (INJ) {
    const float* src = (s == 0) ? a.inj_z0 + (size_t)f * a.J * N
                                : a.inj_z + (((size_t)f * a.T + (s - 1)) * a.J) * N;
#pragma unroll
    for (int e = 0; e < G; ++e)
#pragma unroll
      for (int r = 0; r < N; ++r) z[e * N + r] = (k0 + e < a.J) ? src[(size_t)(k0 + e) * N + r] : 0.0f;
  } else {
    const uint64_t seed = a.seeds[f];
    const uint32_t c0 = (uint32_t)k0 * N / 4;
#pragma unroll
    for (int c = 0; c < G * N / 4; ++c) {
      if (FAST) pp_normal4_fast(seed, c0 + c, (uint32_t)s, PPF_TAG_PROCESS, z + 4 * c);
      else pp_normal4(seed, c0 + c, (uint32_t)s, PPF_TAG_PROCESS, z + 4 * c);
    }
  }
}

__device__ __forceinline__ uint32_t resample_u32(const Args& a, int f, int t) {
  if (a.flags & PPF_F_INJECT) return pp_u32_from_float(a.inj_u[(size_t)f * a.T + t]);
  return pp_resample_u32(a.seeds[f], (uint32_t)(t + 1));
}

// Observation t of series u into registers.
template <class M>
struct Obs {
  float y[M::MAXDY];
  float yc;
  __device__ __forceinline__ void load(const Args& a, int u, int t) {
    const float* p = a.ys + ((size_t)u * a.T + t) * a.model.dy;
#pragma unroll
    for (int i = 0; i < M::MAXDY; ++i) y[i] = (i < a.model.dy) ? p[i] : 0.0f;
    yc = a.ycon ? a.ycon[(size_t)u * a.T + t] : 0.0f;
  }
};

// rproc with the given normals, then dmeas at the loaded observation.
template <class M>
__device__ __forceinline__ float step1(const typename M::Consts& c, const Obs<M>& ob, float* x,
                                       const float* z) {
  M::rproc(c, x, z);
  return M::dmeas(c, ob.y, ob.yc, x);
}

// rproc with the given normals, then dmeas at observation t.
template <class M>
__device__ __forceinline__ float prop1(const Args& a, const typename M::Consts& c, int u, int t,
                                       float* x, const float* z) {
  Obs<M> ob;
  ob.load(a, u, t);
  return step1<M>(c, ob, x, z);
}

// Single-particle propagate into observation t (plain path).
template <class M>
__device__ __forceinline__ float propagate(const Args& a, const typename M::Consts& c, int f, int u,
                                           int j, int t, float* x) {
  float z[M::NZ > 0 ? M::NZ : 1];
  step_noise<M>(a, f, j, t + 1, M::NZ, z);
  return prop1<M>(a, c, u, t, x, z);
}

// Finalise one observation of one filter: log-likelihood term and outputs.
__device__ __forceinline__ void finalize_step(const Args& a, int f, int t, const Acc& acc, uint64_t tot, double* loglik) {
  const bool nanf = acc.nan != 0;
  const float Mx = keyf(acc.maxkey);
  const bool collapsed = !nanf && Mx == -INFINITY;
  double ll;
  if (nanf) ll = __longlong_as_double(0x7ff8000000000000ll);
  else if (collapsed) ll = -INFINITY;
  else ll = (double)Mx + log((double)tot) - 40.0 * kLn2 - (a.mode == MODE_MOP ? log((double)a.J) : 0.0);
  *loglik += ll;
  if ((a.flags & PPF_F_CLL) && a.cll) a.cll[(size_t)f * a.T + t] = ll;
  if (a.mop_M) {
    a.mop_M[(size_t)f * a.T + t] = Mx;
    a.mop_S[(size_t)f * a.T + t] = (double)tot * 9.094947017729282e-13;
  }
  const double S1 = (double)tot * 9.094947017729282e-13;  // 2^-40
  if ((a.flags & PPF_F_ESS) && a.ess) {
    float e;
    if (nanf) e = __int_as_float(0x7fc00000);
    else if (collapsed) e = (float)a.J;
    else e = (float)(S1 * S1 / acc.s2);
    a.ess[(size_t)f * a.T + t] = e;
  }
  // static indices into acc (bounded by dx at run time), so a caller's local
  // record can stay in registers
  const int dx = a.model.dx;
  if ((a.flags & PPF_F_FMEAN) && a.fmean)
#pragma unroll
    for (int d = 0; d < kMaxDim; ++d)
      if (d < dx) a.fmean[((size_t)f * a.T + t) * dx + d] = (float)(collapsed ? acc.px[d] / a.J : acc.fx[d] / S1);
  if ((a.flags & PPF_F_PMEAN) && a.pmean)
#pragma unroll
    for (int d = 0; d < kMaxDim; ++d)
      if (d < dx) a.pmean[((size_t)f * a.T + t) * dx + d] = (float)(acc.px[d] / a.J);
}

__device__ __forceinline__ bool decide_resample(const Args& a, const Acc& acc) {
  if (acc.nan) return false;
  const float Mx = keyf(acc.maxkey);
  if (Mx == -INFINITY) return 0.0f > a.logthresh;
  const float mn = keyf(acc.minkey);
  return (Mx - mn) > a.logthresh;
}

__device__ __forceinline__ void accum_maxmin(float w, unsigned int& mx, unsigned int& mn, unsigned int& nn) {
  const bool bad = (w != w) | (w == INFINITY);
  const unsigned int k = fkey(w);
  nn |= bad ? 1u : 0u;
  mx = bad ? mx : max(mx, k);
  mn = bad ? mn : min(mn, k);
}

// Constants of the exact systematic-offset test for one filter and step:
//   child k lies below CDF value C  <=>  k tot + chi < C J,
// chi = floor(u32 tot / 2^32) (derivation in ppf_core.cuh, nchild).
struct Offsets {
  uint64_t tot, chi;
  double inv, chi_d;   // about J / tot and chi / tot, for the first guess
  int J;
};

// The guess needs no division: 1 / tot from the correctly rounded float
// reciprocal of (float)tot has a relative error below 2^-22, so
// C * J / tot - chi / tot (at most J <= 2^21) is off by less than 1/2 and
// nchild_fast's exact comparisons settle the answer within one step.
__device__ __forceinline__ Offsets make_offsets(uint64_t tot, uint32_t u32, int J) {
  Offsets o;
  o.tot = tot;
  o.chi = __umul64hi((uint64_t)u32 << 32, tot);   // (u32 * tot) >> 32
  const double r = (double)__frcp_rn((float)tot);
  o.inv = (double)J * r;
  o.chi_d = (double)o.chi * r;
  o.J = J;
  return o;
}

// 128-bit a*b for 64-bit a, b as (hi, lo).
__device__ __forceinline__ void mul64(uint64_t a, uint64_t b, uint64_t& hi, uint64_t& lo) {
  lo = a * b;
  hi = __umul64hi(a, b);
}

// nchild(C) = #{ k in [0,J) : k tot + chi < C J } = #{ k : k tot < D },
// D = C J - chi.  The guess ceil(C inv - chi_d) is within one of the answer
// (make_offsets), so one exact 128-bit comparison on each side settles it; a
// bounded loop covers the impossible case defensively.
__device__ __forceinline__ bool lt128(uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl) {
  return (ah < bh) | ((ah == bh) & (al < bl));
}

__device__ __forceinline__ int nchild_fast(const Offsets& o, uint64_t C) {
  uint64_t Dh, Dl;
  mul64(C, (uint64_t)o.J, Dh, Dl);
  Dh -= (Dl < o.chi);
  Dl -= o.chi;                                  // D = C J - chi (may be negative)
  const bool nonpos = ((long long)Dh < 0) | ((Dh == 0) & (Dl == 0));
  long long k = (long long)ceil((double)C * o.inv - o.chi_d);
  k = k < 0 ? 0 : (k > o.J ? o.J : k);
  uint64_t Ph, Pl;
  mul64((uint64_t)k, o.tot, Ph, Pl);            // P = k tot
  for (int it = 0; it < 4; ++it) {
    const uint64_t ql = Pl - o.tot, qh = Ph - (Pl < o.tot);     // (k-1) tot
    const bool down = (k > 0) & !lt128(qh, ql, Dh, Dl);        // (k-1) tot >= D
    const bool up = (k < o.J) & lt128(Ph, Pl, Dh, Dl);          // k tot < D
    if (!(down | up)) break;
    if (down) { Ph = qh; Pl = ql; --k; }
    else { const uint64_t nl = Pl + o.tot; Ph += (nl < Pl); Pl = nl; ++k; }
  }
  return nonpos ? 0 : (int)k;
}

// Incremental form for consecutive parents: with P = k tot + chi and
// D = C J, a parent of weight q moves D by q J (< 2^62) and its children are
// the points P < D passed while advancing k.  No floating point, no division
// for the usual parent of a few children.
struct OffWalk {
  uint64_t Dh, Dl, Ph, Pl;
  int k;
};

__device__ __forceinline__ void offwalk_set_k(const Offsets& o, OffWalk& w, int k) {
  w.k = k;
  mul64((uint64_t)k, o.tot, w.Ph, w.Pl);
  w.Pl += o.chi;
  w.Ph += (w.Pl < o.chi);
}

__device__ __forceinline__ OffWalk offwalk_init(const Offsets& o, uint64_t C) {
  OffWalk w;
  mul64(C, (uint64_t)o.J, w.Dh, w.Dl);
  offwalk_set_k(o, w, nchild_fast(o, C));
  return w;
}

// Add a parent of weight q; returns nchild of the new cumulative weight.
__device__ __forceinline__ int offwalk_add(const Offsets& o, OffWalk& w, uint64_t q) {
  const uint64_t add = q * (uint64_t)o.J;
  w.Dl += add;
  w.Dh += (w.Dl < add);
  while (w.k < o.J && lt128(w.Ph, w.Pl, w.Dh, w.Dl)) {
    w.Pl += o.tot;
    w.Ph += (w.Pl < o.tot);
    ++w.k;
  }
  return w.k;
}

// The points are tot apart, so a parent with q J <= n tot has at most n
// children.  offwalk_add walks them point by point: cheap for the usual parent
// of a few children, but a parent that takes much of the swarm under
// degenerate weights would cost its thread one step per child while the rest
// of the CTA waits.  The callers therefore take the closed form (nchild_fast,
// the same exact count, about as costly as 16 steps) for runs or parents that
// hold more than about 64 expected children:
//   * runs of parents held in registers test the run first (run_has_heavy,
//     run_has_heavy_e) and then either walk (the usual case, the same code as
//     without the test) or evaluate every offset in closed form;
//   * loops over parents in shared or global memory call offwalk_add_c,
//     which keeps the cumulative weight C (D = C J) and jumps per parent.
// Both forms are exact, so the threshold only picks the faster one.
__device__ __forceinline__ bool heavy_parent(const Offsets& o, uint64_t q) {
  return ((q * (uint64_t)o.J) >> 6) > o.tot;
}
template <int N>
__device__ __forceinline__ bool run_has_heavy(const Offsets& o, const uint64_t (&q)[N]) {
  uint64_t m = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) m = q[i] > m ? q[i] : m;
  return heavy_parent(o, m);
}
// The same test on the float weights e = q 2^-40 (an estimate is enough).
template <int N>
__device__ __forceinline__ bool run_has_heavy_e(const float (&e)[N], uint64_t tot, int J) {
  float m = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) m = fmaxf(m, e[i]);
  return m * (float)J > (float)tot * (64.0f / 1099511627776.0f);
}
__device__ __forceinline__ int offwalk_add_c(const Offsets& o, OffWalk& w, uint64_t& C, uint64_t q) {
  C += q;
  if (heavy_parent(o, q)) {
    const uint64_t add = q * (uint64_t)o.J;
    w.Dl += add;
    w.Dh += (w.Dl < add);
    offwalk_set_k(o, w, nchild_fast(o, C));
    return w.k;
  }
  return offwalk_add(o, w, q);
}

// Parent (tile-local index) of child k: the last l in [0, n) with st[l] <= k.
__device__ __forceinline__ int find_parent(const int* st, int n, int k) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (st[mid] <= k) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ============================================================================
// STREAM path
// ============================================================================

// Per-filter model constants, computed once per call (Cholesky factors, log
// determinants, transformed parameters) and copied by every block.
// Bytes per filter in the workspace: M::CONST_BYTES (512, or 2048 for the
// wide LG); the workspace reserves const_bytes(model) per filter.
template <class M>
__global__ void k_prep(Args a) {
  static_assert(sizeof(typename M::Consts) <= M::CONST_BYTES, "Consts stride");
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.F) return;
  typename M::Consts c;
  M::prepare(c, a.theta + (size_t)f * a.model.n_params, a.model, (a.flags & PPF_F_EST) != 0);
  *reinterpret_cast<typename M::Consts*>(a.consts + (size_t)f * M::CONST_BYTES) = c;
}

template <class M>
__device__ __forceinline__ void load_consts(const Args& a, int f, typename M::Consts& c) {
  constexpr int NW = (sizeof(typename M::Consts) + 3) / 4;
  const uint32_t* src = reinterpret_cast<const uint32_t*>(a.consts + (size_t)f * M::CONST_BYTES);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&c);
  for (int i = threadIdx.x; i < NW; i += blockDim.x) dst[i] = src[i];
}

// Store the 4 children k0..k0+3 (valid[e]) of one group: float4 stores when
// the whole group is valid and rows are 16-byte aligned (J % 4 == 0).
template <int DX>
__device__ __forceinline__ void store_group(float* Xn, float* Wn, float* logw, int J, int k0,
                                            const float (&xo)[4][DX], const float (&wo)[4],
                                            int nvalid_lo, int nvalid_hi) {
  const bool full = (nvalid_lo == 0) & (nvalid_hi == 4) & ((J & 3) == 0);
  if (full) {
#pragma unroll
    for (int d = 0; d < DX; ++d)
      *reinterpret_cast<float4*>(Xn + d * J + k0) = make_float4(xo[0][d], xo[1][d], xo[2][d], xo[3][d]);
    *reinterpret_cast<float4*>(Wn + k0) = make_float4(wo[0], wo[1], wo[2], wo[3]);
    if (logw) *reinterpret_cast<float4*>(logw + k0) = make_float4(wo[0], wo[1], wo[2], wo[3]);
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (e < nvalid_lo || e >= nvalid_hi) continue;
#pragma unroll
      for (int d = 0; d < DX; ++d) Xn[d * J + k0 + e] = xo[e][d];
      Wn[k0 + e] = wo[e];
      if (logw) logw[k0 + e] = wo[e];
    }
  }
}


// Store the G children k0..k0+G-1 (valid in [lo, hi)): one vector store per
// row when the whole group is valid and the rows are aligned to G floats.
template <int G, int DX>
__device__ __forceinline__ void store_group_g(float* Xn, float* Wn, float* logw, int J, int k0,
                                              const float (&xo)[G][DX], const float (&wo)[G], int lo, int hi) {
  if (G == 4) {
    store_group<DX>(Xn, Wn, logw, J, k0, reinterpret_cast<const float(&)[4][DX]>(xo),
                    reinterpret_cast<const float(&)[4]>(wo), lo, hi);
    return;
  }
  const bool full = (lo == 0) & (hi == G) & ((J & (G - 1)) == 0);
  if (G == 2 && full) {
#pragma unroll
    for (int d = 0; d < DX; ++d)
      *reinterpret_cast<float2*>(Xn + d * J + k0) = make_float2(xo[0][d], xo[G > 1 ? 1 : 0][d]);
    *reinterpret_cast<float2*>(Wn + k0) = make_float2(wo[0], wo[G > 1 ? 1 : 0]);
    if (logw) *reinterpret_cast<float2*>(logw + k0) = make_float2(wo[0], wo[G > 1 ? 1 : 0]);
    return;
  }
#pragma unroll
  for (int e = 0; e < G; ++e) {
    if (e < lo || e >= hi) continue;
#pragma unroll
    for (int d = 0; d < DX; ++d) Xn[d * J + k0 + e] = xo[e][d];
    Wn[k0 + e] = wo[e];
    if (logw) logw[k0 + e] = wo[e];
  }
}

// ------------------------------ IF2 helpers --------------------------------
// (shared by the streaming IF2 kernels, ppf_if2.cu, and the cluster kernels,
// ppf_cluster.cu)

// jnp.nan_to_num(m, nan=log(1e-18)): NaN -> log(1e-18), +inf -> FLT_MAX,
// -inf -> -FLT_MAX.
__device__ __forceinline__ float if2_measure(float m, float log1e18) {
  if (m != m) return log1e18;
  if (m == INFINITY) return FLT_MAX;
  if (m == -INFINITY) return -FLT_MAX;
  return m;
}

// Perturb the parameter row th[0..P) of particle k in place:
// th[p] += (cool * sig[p]) * z_p, z_p the P normals of counter s (tag PERTURB),
// drawn one at a time from the particle's Philox blocks (the same values
// pp_normals gives), or read from the injected arrays.  The row lives in
// shared memory: per-thread arrays passed by pointer and indexed at run time
// are kept out of these kernels.
template <bool INJ>
__device__ __forceinline__ void perturb_row(const Args& a, int f, int k, int s, int P, float cool,
                                            const float* sig, float* th) {
  if (INJ) {
    const float* src = (s == 0) ? a.inj_zp0 + ((size_t)f * a.J + k) * P
                                : a.inj_zp + (((size_t)f * a.T + (s - 1)) * a.J + k) * P;
    for (int p = 0; p < P; ++p) th[p] = th[p] + (cool * sig[p]) * src[p];
    return;
  }
  const uint64_t seed = a.seeds[f];
  uint32_t cached = 0xffffffffu;
  float z4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int p = 0; p < P; ++p) {
    const uint32_t i = (uint32_t)k * (uint32_t)P + (uint32_t)p;
    if ((i >> 2) != cached) {
      cached = i >> 2;
      pp_normal4(seed, cached, (uint32_t)s, PPF_TAG_PERTURB, z4);
    }
    const uint32_t e = i & 3u;
    const float z = e == 0u ? z4[0] : e == 1u ? z4[1] : e == 2u ? z4[2] : z4[3];
    th[p] = th[p] + (cool * sig[p]) * z;
  }
}

// Parameter rows of the block's threads in dynamic shared memory: thread r
// owns row r, stride P | 1 (odd, so a warp's rows fall in distinct banks).
__device__ __forceinline__ int if2_row_stride(int P) { return P | 1; }

// Fixed-point sums of the weights of one tile, published as the tile's total
// in desc[t & 1].  The body for tile b of filter f at step t.
// SCAN = true (k_sum, one launch per step): each tile publishes its total and
// counts itself done (a fence, then an atomic on the filter's counter); the
// tile that finds every other tile of its filter already done forms all the
// filter's exclusive tile prefixes and its total (excl, tot) for the next
// kernel.  No tile waits on another, and the prefixes are exact integer sums,
// so they do not depend on which tile finishes last.
// SCAN = false (the persistent MOP forward, all tiles resident and a grid
// barrier after this body): the prefix is left to tile_prefix.
template <class M, int TPB, int IT, bool SCAN = true, bool FAST = false>
__device__ __forceinline__ void sum_tile(const Args& a, int t, int f, int b) {
  constexpr int TILE = TPB * IT;
  constexpr int DX = M::MAXDX;
  __shared__ uint64_t s_red[TPB / 32];
  __shared__ double sd[TPB / 32];
  const int u = filter_unit(a, f);
  if (t >= filter_len(a, u)) return;
  const int p = t & 1;
  const Acc& acc = a.acc[p][f];   // read in place (a copy would sit in local memory)
  if (b == 0 && threadIdx.x == 0) {
    Acc* nx = a.acc[p ^ 1] + f;
    nx->maxkey = 0u; nx->minkey = 0xffffffffu; nx->nan = 0u;
    nx->s2 = 0.0;
    for (int d = 0; d < kMaxDim; ++d) { nx->fx[d] = 0.0; nx->px[d] = 0.0; }
  }
  const bool nanf = acc.nan != 0;
  const float Mx = keyf(acc.maxkey);
  const bool collapsed = nanf || Mx == -INFINITY;
  const int J = a.J;
  float* W = a.W[p] + (size_t)f * J;
  const int jb = b * TILE + threadIdx.x * IT;
  const bool vec = jb + IT <= J && (IT % 4) == 0 && (J & 3) == 0;
  uint64_t qs = 0;
  float wv[IT], ev[IT];
  // float4 loads only when every filter's row starts 16-byte aligned (J % 4 == 0)
  if (vec) {
#pragma unroll
    for (int i = 0; i < IT; i += 4) {
      const float4 v4 = *reinterpret_cast<const float4*>(W + jb + i);
      wv[i] = v4.x; wv[i + 1] = v4.y; wv[i + 2] = v4.z; wv[i + 3] = v4.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < IT; ++i) wv[i] = (jb + i < J) ? W[jb + i] : -INFINITY;
  }
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    ev[i] = qweight_e_t<FAST>(wv[i], Mx, collapsed);
    qs += (jb + i < J) ? qweight_from_e(ev[i]) : 0ull;
  }
  // a resampling step reads its parents' weights only through q: keep e in
  // their place for k_resprop (the step's carried weights need the originals)
  const bool rs = decide_resample(a, acc);
  if (rs) {
    if (vec) {
#pragma unroll
      for (int i = 0; i < IT; i += 4)
        *reinterpret_cast<float4*>(W + jb + i) = make_float4(ev[i], ev[i + 1], ev[i + 2], ev[i + 3]);
    } else {
#pragma unroll
      for (int i = 0; i < IT; ++i)
        if (jb + i < J) W[jb + i] = ev[i];
    }
  }
  // block scan: the tile total, and on a resampling step each thread's
  // exclusive prefix for k_resprop (its threads own the same runs of parents)
  // (one barrier: warp scans, then every thread adds the totals of the warps
  // before its own; s_red is not reused, so no trailing barrier)
  uint64_t btot = 0;
  {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t inc = warp_incl_scan_u64(qs);
    if (lane == 31) s_red[warp] = inc;
    __syncthreads();
    uint64_t before = 0;
#pragma unroll
    for (int w = 0; w < TPB / 32; ++w) {
      const uint64_t v = s_red[w];
      before += (w < warp) ? v : 0ull;
      btot += v;
    }
    if (rs) a.runpre[((size_t)f * a.ntiles + b) * TPB + threadIdx.x] = before + inc - qs;
  }
  uint64_t* desc = a.desc[p] + (size_t)f * a.ntiles;
  if (threadIdx.x == 0) desc[b] = btot;
  if (SCAN) {
    __shared__ int s_last;
    __shared__ uint64_t s_scan2[TPB / 32 + 1];
    if (threadIdx.x == 0) {
      __threadfence();   // the total is visible before the count that reveals it
      s_last = atomicAdd(a.fdone[p] + f, 1u) == (unsigned int)(a.ntiles - 1);
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      // every thread sums a run of consecutive tile totals; one block scan of
      // the runs, then each tile's exclusive prefix along the run
      const int nt = a.ntiles;
      const int per = (nt + TPB - 1) / TPB;
      const int i0 = min(nt, (int)threadIdx.x * per), i1 = min(nt, i0 + per);
      uint64_t run = 0;
      for (int i = i0; i < i1; ++i) run += __ldcg(reinterpret_cast<const unsigned long long*>(desc + i));
      uint64_t all;
      uint64_t pre = block_excl_scan_u64_1b<TPB>(run, s_scan2, all);
      uint64_t* ex = a.excl + (size_t)f * nt;
      for (int i = i0; i < i1; ++i) {
        ex[i] = pre;
        pre += __ldcg(reinterpret_cast<const unsigned long long*>(desc + i));
      }
      if (threadIdx.x == 0) a.tot[f] = all;
    }
  }
  if (a.flags & PPF_F_ESS) {
    double s2 = 0.0;
#pragma unroll
    for (int i = 0; i < IT; ++i)
      if (jb + i < J) {
        const double e = collapsed ? 1.0 : (double)pp_expf(wv[i] - Mx);
        s2 += e * e;
      }
    const double s = block_sum_f64<TPB>(s2, sd);
    if (threadIdx.x == 0) atomicAdd(&a.acc[p][f].s2, s);
  }
  if (a.flags & PPF_F_FMEAN) {
    const float* X = a.X[p] + (size_t)f * DX * J;
#pragma unroll
    for (int d = 0; d < DX; ++d) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < IT; ++i)
        if (jb + i < J) {
          const double e = collapsed ? 1.0 : (double)pp_expf(wv[i] - Mx);
          s += (double)X[d * J + jb + i] * e;
        }
      s = block_sum_f64<TPB>(s, sd);
      if (threadIdx.x == 0) atomicAdd(&a.acc[p][f].fx[d], s);
    }
  }
}

// After sum_tile<..., false> on every tile and a grid barrier: tile b's
// exclusive prefix and the filter's total from the published tile totals
// (every CTA of the filter writes the same total).
__device__ __forceinline__ void tile_prefix(const Args& a, int t, int f, int b) {
  if (threadIdx.x < 32) {
    const uint64_t* sums = a.desc[t & 1] + (size_t)f * a.ntiles;
    uint64_t before = 0, all = 0;
    for (int i = threadIdx.x; i < a.ntiles; i += 32) {
      const uint64_t v = sums[i];
      all += v;
      before += (i < b) ? v : 0ull;
    }
    before = warp_sum_u64(before);
    all = warp_sum_u64(all);
    if (threadIdx.x == 0) {
      a.excl[(size_t)f * a.ntiles + b] = before;
      a.tot[f] = all;
    }
  }
  __syncthreads();
}

// One CTA per tile: fixed-point weights, e in place, run prefixes and the
// tile total; the filter's last tile forms the tile prefixes (sum_tile).
template <class M, int TPB, int IT>
__global__ void __launch_bounds__(TPB) k_sum(Args a, int t) {
  const int v = blockIdx.x;
  sum_tile<M, TPB, IT, true>(a, t, v / a.ntiles, v % a.ntiles);
}

}  // namespace ppf
