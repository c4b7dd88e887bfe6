// ppf_if2.cu -- one iteration of IF2's perturbed particle filter.
//
// Replaces _perfilter_internal / _perfilter_scan_body
// (pypomp/core/algorithms/mif.py:88-258) and _resampler_thetas
// (helpers.py:103-141): every particle carries its own parameter vector on
// the estimation scale.  Before the first step the vector is perturbed with
// sds rw_sig0 * cool0 (mif.py:113-120) and the initial state is drawn with it;
// before every step it is perturbed with sds rw_sig * cool[t] (mif.py:178-181),
// then rproc and dmeas run with the perturbed vector, non-finite measurement
// densities are mapped as jnp.nan_to_num(..., nan=log(1e-18)) does
// (mif.py:205-210), and resampling moves state and vector together.  The
// output is the swarm after the final resampling and the log-likelihood.
// Weights, the exact CDF and the systematic offsets are those of the bootstrap
// filter (the same k_sum, the same offset walk).
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "ppf.h"
#include "ppf_core.cuh"
#include "ppf_internal.h"
#include "ppf_kernels.cuh"
#include "ppf_models.cuh"

namespace ppf {

template <class M, int TPB, bool INJ>
__global__ void __launch_bounds__(TPB) k_if2_init(Args a) {
  extern __shared__ __align__(16) float s_rows[];   // [TPB][P | 1]
  __shared__ unsigned int smk[2 * (TPB / 32)];
  constexpr int DX = M::MAXDX;
  const int f = blockIdx.y;
  const int u = filter_unit(a, f);
  const int J = a.J, P = a.model.n_params;
  const float log1e18 = pp_logf(1e-18f);
  Obs<M> ob;
  ob.load(a, u, 0);
  const float c0 = a.cool0[u], c1 = a.cool[(size_t)u * a.T];
  float* X = a.X[0] + (size_t)f * DX * J;
  float* W = a.W[0] + (size_t)f * J;
  float* TH = a.TH[0] + (size_t)f * P * J;
  const float* S = a.swarm_in + (size_t)f * P * J;
  float* th = s_rows + threadIdx.x * if2_row_stride(P);
  unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
  const int k = blockIdx.x * TPB + threadIdx.x;
  if (k < J) {
    for (int p = 0; p < P; ++p) th[p] = S[(size_t)p * J + k];
    perturb_row<INJ>(a, f, k, 0, P, c0, a.rw_sig0, th);
    typename M::Consts c;
    M::prepare(c, th, a.model, (a.flags & PPF_F_EST) != 0);
    float x[DX];
    float z0[M::NZ0 > 0 ? M::NZ0 : 1];
    step_noise<M>(a, f, k, 0, M::NZ0, z0);
    M::rinit(c, z0, x);
    perturb_row<INJ>(a, f, k, 1, P, c1, a.rw_sig, th);
    M::prepare(c, th, a.model, (a.flags & PPF_F_EST) != 0);
    float z[M::NZ];
    step_noise<M>(a, f, k, 1, M::NZ, z);
    const float m = if2_measure(step1<M>(c, ob, x, z), log1e18);
    const float w = a.base_init + m;
#pragma unroll
    for (int d = 0; d < DX; ++d) X[d * J + k] = x[d];
    W[k] = w;
    for (int p = 0; p < P; ++p) TH[(size_t)p * J + k] = th[p];
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
}

// Resample the tile's parents (state + parameter vector) and, unless this is
// the filter's last step, perturb each child's vector and propagate it.
// Parent states are staged in shared memory; a child reads its parent's
// parameter vector straight from global memory (children of consecutive
// parents are consecutive, so a warp's reads stay nearly coalesced).
template <class M, int TPB, int IT, bool INJ>
__global__ void __launch_bounds__(TPB) k_if2_resprop(Args a, int t) {
  constexpr int TILE = TPB * IT;
  constexpr int DX = M::MAXDX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int P = a.model.n_params;
  float* xs = reinterpret_cast<float*>(smem_raw);                 // [DX][TILE]
  int* st = reinterpret_cast<int*>(xs + DX * TILE);               // [TILE + 1]
  float* wcar = reinterpret_cast<float*>(st + TILE + 4);          // [TILE]
  float* th = wcar + TILE + threadIdx.x * if2_row_stride(P);      // [TPB][P | 1]
  __shared__ unsigned int smk[2 * (TPB / 32)];

  const int f = blockIdx.y, b = blockIdx.x;
  const int u = filter_unit(a, f);
  const int Tf = filter_len(a, u);
  const int p2 = t & 1;
  if (threadIdx.x == 0) {
    a.desc[p2 ^ 1][(size_t)f * a.ntiles + b] = 0ull;
    if (b == 0 && f == 0) a.counter[p2 ^ 1] = 0;
    if (b == 0) a.fdone[p2 ^ 1][f] = 0u;   // the next step's tile count
  }
  if (t >= Tf) return;
  const Acc& acc = a.acc[p2][f];   // read in place (a copy would sit in local memory)
  const uint64_t tot = a.tot[f];
  if (b == 0 && threadIdx.x == 0) finalize_step(a, f, t, acc, tot, a.loglik + f);
  const bool last = (t == Tf - 1);
  const bool nanf = acc.nan != 0;
  const float Mx = keyf(acc.maxkey);
  const bool collapsed = !nanf && Mx == -INFINITY;
  const bool rs = decide_resample(a, acc);
  const int J = a.J;
  const int jt = b * TILE;
  const int ntile = min(TILE, J - jt);
  const float* Xc = a.X[p2] + (size_t)f * DX * J;
  const float* Wc = a.W[p2] + (size_t)f * J;
  const float* THc = a.TH[p2] + (size_t)f * P * J;
  float* Xn = a.X[p2 ^ 1] + (size_t)f * DX * J;
  float* Wn = a.W[p2 ^ 1] + (size_t)f * J;
  float* THn = a.TH[p2 ^ 1] + (size_t)f * P * J;
  float* Sout = a.swarm_out + (size_t)f * P * J;
  int* anc = a.anc ? a.anc + ((size_t)f * a.T + t) * J : nullptr;
  const float log1e18 = pp_logf(1e-18f);
  Obs<M> ob;
  if (!last) ob.load(a, u, t + 1);
  const float cl = last ? 0.0f : a.cool[(size_t)u * a.T + t + 1];
  const int l0 = threadIdx.x * IT;
  {
    float wv[IT];
#pragma unroll
    for (int i = 0; i < IT; ++i) wv[i] = (l0 + i < ntile) ? Wc[jt + l0 + i] : 0.0f;
    if (rs) {
      const Offsets o = make_offsets(tot, resample_u32(a, f, t), J);
      const uint64_t E = a.excl[(size_t)f * a.ntiles + b];
      uint64_t q[IT];
#pragma unroll
      for (int i = 0; i < IT; ++i) q[i] = (l0 + i < ntile) ? qweight_from_e(wv[i]) : 0ull;   // k_sum left e
      // the exclusive prefix of this thread's run within the tile, from k_sum
      const uint64_t tex = a.runpre[((size_t)f * a.ntiles + b) * TPB + threadIdx.x];
      if (l0 < ntile && !run_has_heavy_e(wv, tot, J)) {
        OffWalk wk = offwalk_init(o, E + tex);
        st[l0] = wk.k;
#pragma unroll
        for (int i = 0; i < IT; ++i) {
          if (l0 + i >= ntile) break;
          const int kn = offwalk_add(o, wk, q[i]);
          if (i + 1 < IT || l0 + i + 1 == ntile) st[l0 + i + 1] = kn;
        }
      } else if (l0 < ntile) {
        uint64_t C = E + tex;   // a heavy parent in the run: closed form throughout
        st[l0] = nchild_fast(o, C);
#pragma unroll
        for (int i = 0; i < IT; ++i) {
          if (l0 + i >= ntile) break;
          C += q[i];
          const int kn = nchild_fast(o, C);
          if (i + 1 < IT || l0 + i + 1 == ntile) st[l0 + i + 1] = kn;
        }
      }
    } else {
      float lt32 = 0.0f;
      if (nanf) lt32 = __int_as_float(0x7fc00000);
      else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
      const float nwc = -pp_logf((float)J);
#pragma unroll
      for (int i = 0; i < IT; ++i)
        if (l0 + i < ntile) {
          st[l0 + i] = jt + l0 + i;
          wcar[l0 + i] = collapsed ? nwc : wv[i] - lt32;
        }
      if (l0 < ntile && l0 + IT >= ntile) st[ntile] = jt + ntile;
    }
  }
  for (int l = threadIdx.x; l < ntile; l += TPB) {
#pragma unroll
    for (int d = 0; d < DX; ++d) xs[d * TILE + l] = Xc[d * J + jt + l];
  }
  __syncthreads();
  const int klo = st[0], khi = st[ntile];
  unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
  for (int k = klo + threadIdx.x; k < khi; k += TPB) {
    const int l = find_parent(st, ntile, k);
    if (anc) anc[k] = jt + l;
    for (int p = 0; p < P; ++p) th[p] = THc[(size_t)p * J + jt + l];
    if (last) {
      for (int p = 0; p < P; ++p) Sout[(size_t)p * J + k] = th[p];
      continue;
    }
    perturb_row<INJ>(a, f, k, t + 2, P, cl, a.rw_sig, th);
    typename M::Consts c;
    M::prepare(c, th, a.model, (a.flags & PPF_F_EST) != 0);
    float x[DX];
#pragma unroll
    for (int d = 0; d < DX; ++d) x[d] = xs[d * TILE + l];
    float z[M::NZ];
    step_noise<M>(a, f, k, t + 2, M::NZ, z);
    const float m = if2_measure(step1<M>(c, ob, x, z), log1e18);
    const float w = (rs ? a.base_rs : wcar[l]) + m;
#pragma unroll
    for (int d = 0; d < DX; ++d) Xn[d * J + k] = x[d];
    Wn[k] = w;
    for (int p = 0; p < P; ++p) THn[(size_t)p * J + k] = th[p];
    accum_maxmin(w, mx, mn, nn);
  }
  if (last) return;
  block_maxmin_u32<TPB>(mx, mn, smk);
  nn = __syncthreads_or(nn);
  Acc* an = a.acc[p2 ^ 1] + f;
  if (threadIdx.x == 0) {
    if (mx) atomicMax(&an->maxkey, mx);
    if (mn != 0xffffffffu) atomicMin(&an->minkey, mn);
    if (nn) atomicOr(&an->nan, 1u);
  }
}

static int if2_row_stride_host(int P) { return P | 1; }

template <class M, int TPB, int IT, bool INJ>
int run_if2_t(Args& a, cudaStream_t s) {
  constexpr int TILE = TPB * IT;
  if (a.tile != TILE || a.ntiles != (a.J + TILE - 1) / TILE) return PPF_EINTERNAL;
  const size_t rows = sizeof(float) * TPB * if2_row_stride_host(a.model.n_params);
  const size_t smem = sizeof(float) * M::MAXDX * TILE + sizeof(int) * (TILE + 4) + sizeof(float) * TILE + rows;
  if (smem > kResidentSmemMax) return PPF_EUNSUPPORTED;
  if (cudaFuncSetAttribute(k_if2_resprop<M, TPB, IT, INJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return PPF_ECUDA;
  if (cudaFuncSetAttribute(k_if2_init<M, TPB, INJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)rows) != cudaSuccess)
    return PPF_ECUDA;
  dim3 grid_init((a.J + TPB - 1) / TPB, a.F);
  dim3 grid(a.ntiles, a.F);
  PROF_BEGIN(KIND_IF2);
  k_if2_init<M, TPB, INJ><<<grid_init, TPB, rows, s>>>(a);
  for (int t = 0; t < a.T; ++t) {
    k_sum<M, TPB, IT><<<a.ntiles * a.F, TPB, 0, s>>>(a, t);
    k_if2_resprop<M, TPB, IT, INJ><<<grid, TPB, smem, s>>>(a, t);
  }
  PROF_END(KIND_IF2);
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M, bool INJ>
int run_if2_tiled(Args& a, cudaStream_t s) {
  switch (a.tile) {
    case kTileLarge: return run_if2_t<M, 256, 8, INJ>(a, s);
    case kTileMid: return run_if2_t<M, 128, 4, INJ>(a, s);
    case kTileSmall: return run_if2_t<M, 64, 4, INJ>(a, s);
    default: return PPF_EINVAL;
  }
}

template <class M>
int run_if2_m(Args& a, cudaStream_t s) {
  if constexpr (M::WIDE) {
    // the wide LG: Philox draws, 256-particle tiles (the per-thread parameter
    // rows of up to 261 entries fit shared memory only with 64 threads)
    if (a.flags & PPF_F_INJECT) return PPF_EUNSUPPORTED;
    return a.tile == kTileSmall ? run_if2_t<M, 64, 4, false>(a, s) : PPF_EINTERNAL;
  } else {
    return (a.flags & PPF_F_INJECT) ? run_if2_tiled<M, true>(a, s) : run_if2_tiled<M, false>(a, s);
  }
}

int run_if2(Args& a, cudaStream_t s) {
  // few small swarms (the unit filters of a panel): one cluster per filter
  // keeps the swarm and its parameter rows on chip for the whole time loop.
  // Measured on Ricker (T = 500): the cluster path wins up to F J = 65536
  // particles in all (J = 8192, F = 8: 8.8 vs 15.0 ms) and loses at 262144
  // (J = 32768, F = 8: 21.4 vs 17.7 ms), where a CTA holds several children
  // per thread of heavy per-particle IF2 work.
  const long long tiles = (long long)a.F * ((a.J + kTileLarge - 1) / kTileLarge);
  if (!(a.flags & PPF_F_NO_CLUSTER) && tiles < 2LL * kNumSMs && (long long)a.F * a.J <= 131072 &&
      cluster_fits(a, true)) {
    const int rc = run_cluster(a, true, s);
    if (rc != PPF_EUNSUPPORTED) return rc;
  }
  switch (a.model.kind) {
        case PPF_MODEL_LG:
      return with_lg<int>(a.model, true, PPF_EUNSUPPORTED,
                          [&](auto tg) { return run_if2_m<typename decltype(tg)::type>(a, s); });
    case PPF_MODEL_SV: return run_if2_m<SV>(a, s);
    case PPF_MODEL_RICKER: return run_if2_m<Ricker>(a, s);
    default: return PPF_EINVAL;
  }
}

}  // namespace ppf
