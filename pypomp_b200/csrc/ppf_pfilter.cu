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
//             k_sum      fixed-point weights, tile totals; the filter's last
//                        tile to finish forms every tile's exclusive prefix
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
#include "ppf_kernels.cuh"
#include "ppf_stream.cuh"

namespace ppf {

template <class M, int TPB, bool INJ>
__global__ void __launch_bounds__(TPB) k_init(Args a) {
  init_tile<M, TPB, INJ>(a, blockIdx.y, blockIdx.x);
}

template <class M, int TPB, int IT, bool INJ>
__global__ void __launch_bounds__(TPB, RespropOccupancy<M>::B * (256 / TPB)) k_resprop(Args a, int t) {
  resprop_tile<M, TPB, IT, INJ, true>(a, t, blockIdx.y, blockIdx.x);
}


// ============================================================================
// RESIDENT path: one CTA per filter, the whole time loop in one launch.
// Shared memory: xs[DX][J] float, ws[J] float, st[J+1] int.  Children are
// processed in runs of 8 per thread and buffered in registers until every
// parent has been read.
// ============================================================================

template <class M, int TPB, int MAXR, bool INJ>
__global__ void __launch_bounds__(TPB, 1) k_resident(Args a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int DX = M::MAXDX;
  constexpr int RUN = 8;
  const int J = a.J;
  float* xs = reinterpret_cast<float*>(smem_raw);
  float* ws = xs + (size_t)DX * J;
  int* st = reinterpret_cast<int*>(ws + J);
  __shared__ typename M::Consts c;
  __shared__ uint64_t s_scan[TPB / 32 + 1];
  __shared__ unsigned int smk[2 * (TPB / 32)];
  __shared__ double sd[TPB / 32];
  __shared__ Acc s_acc;
  __shared__ double s_ll;

  const int f = blockIdx.x;
  const int u = filter_unit(a, f);
  const int Tf = filter_len(a, u);
  if (threadIdx.x == 0) {
    M::prepare(c, a.theta + (size_t)f * a.model.n_params, a.model, (a.flags & PPF_F_EST) != 0);
    s_ll = 0.0;
  }
  __syncthreads();
  const typename M::Consts cr = c;
  // blocked ownership for the scan: thread owns [l0, l1)
  const int per = (J + TPB - 1) / TPB;
  const int l0 = min(J, threadIdx.x * per);
  const int l1 = min(J, l0 + per);

  // step 0: rinit + rproc + dmeas, groups of 4
  Obs<M> ob;
  ob.load(a, u, 0);
  for (int g = threadIdx.x; 4 * g < J; g += TPB) {
    const int k0 = 4 * g;
    float z0[4 * (M::NZ0 > 0 ? M::NZ0 : 1)];
    float z[4 * M::NZ];
    group_noise<M::NZ0, INJ>(a, f, 0, k0, z0);
    group_noise<M::NZ, INJ>(a, f, 1, k0, z);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = k0 + e;
      if (k >= J) break;
      float x[DX];
      M::rinit(cr, z0 + e * M::NZ0, x);
      const float w = (a.mode == MODE_MOP ? 0.0f : a.base_init) + step1<M>(cr, ob, x, z + e * M::NZ);
#pragma unroll
      for (int d = 0; d < DX; ++d) xs[d * J + k] = x[d];
      ws[k] = w;
      if (a.logw) a.logw[((size_t)f * a.T) * J + k] = w;
    }
  }
  __syncthreads();
  const float base = (a.mode == MODE_MOP) ? 0.0f : a.base_rs;

  for (int t = 0; t < Tf; ++t) {
    // (a) max / min / nan
    unsigned int mx = 0u, mn = 0xffffffffu, nn = 0u;
    for (int j = l0; j < l1; ++j) accum_maxmin(ws[j], mx, mn, nn);
    block_maxmin_u32<TPB>(mx, mn, smk);
    nn = __syncthreads_or(nn);
    if (threadIdx.x == 0) {
      s_acc.maxkey = mx; s_acc.minkey = mn; s_acc.nan = nn; s_acc.s2 = 0.0;
      for (int d = 0; d < DX; ++d) { s_acc.fx[d] = 0.0; s_acc.px[d] = 0.0; }
    }
    __syncthreads();
    const bool nanf = s_acc.nan != 0;
    const float Mx = keyf(s_acc.maxkey);
    const bool collapsed = !nanf && Mx == -INFINITY;
    const bool qc = nanf || Mx == -INFINITY;
    // (b) fixed-point weights, scan, total
    uint64_t qs = 0;
    for (int j = l0; j < l1; ++j) qs += qweight(ws[j], Mx, qc);
    uint64_t tot;
    const uint64_t tex = block_excl_scan_u64<TPB>(qs, s_scan, tot);
    if (a.flags & PPF_F_ESS) {
      double s2 = 0.0;
      for (int j = l0; j < l1; ++j) {
        const double e = qc ? 1.0 : (double)pp_expf(ws[j] - Mx);
        s2 += e * e;
      }
      const double s = block_sum_f64<TPB>(s2, sd);
      if (threadIdx.x == 0) s_acc.s2 = s;
    }
    if (a.flags & (PPF_F_FMEAN | PPF_F_PMEAN)) {
#pragma unroll
      for (int d = 0; d < DX; ++d) {
        double sf = 0.0, sp = 0.0;
        for (int j = l0; j < l1; ++j) {
          const double xv = (double)xs[d * J + j];
          sp += xv;
          sf += xv * (qc ? 1.0 : (double)pp_expf(ws[j] - Mx));
        }
        sf = block_sum_f64<TPB>(sf, sd);
        sp = block_sum_f64<TPB>(sp, sd);
        if (threadIdx.x == 0) { s_acc.fx[d] = sf; s_acc.px[d] = sp; }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double ll = s_ll;
      finalize_step(a, f, t, s_acc, tot, &ll);
      s_ll = ll;
    }
    const bool last = (t == Tf - 1);
    if (last && !a.anc) break;
    const bool rs = decide_resample(a, s_acc);
    int* anc = a.anc ? a.anc + ((size_t)f * a.T + t) * J : nullptr;
    float* logw = a.logw ? a.logw + ((size_t)f * a.T + t + 1) * J : nullptr;
    if (!last) ob.load(a, u, t + 1);
    // (c) first-child offsets of every parent (identity without resampling);
    //     without resampling the carried weight replaces ws in place
    if (rs) {
      const Offsets o = make_offsets(tot, resample_u32(a, f, t), J);
      if (l0 < l1) {
        uint64_t C = tex;
        OffWalk wk = offwalk_init(o, C);
        for (int j = l0; j < l1; ++j) {
          st[j] = wk.k;
          offwalk_add_c(o, wk, C, qweight(ws[j], Mx, qc));
        }
      }
    } else {
      float lt32 = 0.0f;
      if (nanf) lt32 = __int_as_float(0x7fc00000);
      else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
      const float nwc = -pp_logf((float)J);
      for (int j = l0; j < l1; ++j) {
        st[j] = j;
        ws[j] = collapsed ? nwc : ws[j] - lt32;
      }
    }
    if (threadIdx.x == TPB - 1) st[J] = J;
    __syncthreads();
    if (J <= 2 * TPB) {
      // (d') few particles: one child per thread at a time, so every thread
      // works (runs of 8 would leave most of them idle and put 8 children on
      // each busy thread's critical path); each child draws its own normals,
      // the same numbers as the grouped draw below
      float cx[2][DX], cw[2];
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) {
        const int k = threadIdx.x + ri * TPB;
        if (k < J) {
          const int l = find_parent(st, J, k);
          if (anc) anc[k] = l;
          float x[DX];
#pragma unroll
          for (int d = 0; d < DX; ++d) x[d] = xs[d * J + l];
          float z[M::NZ];
          if (!last) step_noise<M>(a, f, k, t + 2, M::NZ, z);
          const float wb = rs ? base : ws[l];
          cw[ri] = last ? 0.0f : wb + step1<M>(cr, ob, x, z);
#pragma unroll
          for (int d = 0; d < DX; ++d) cx[ri][d] = x[d];
        }
      }
      __syncthreads();
      if (last) break;
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) {
        const int k = threadIdx.x + ri * TPB;
        if (k < J) {
#pragma unroll
          for (int d = 0; d < DX; ++d) xs[d * J + k] = cx[ri][d];
          ws[k] = cw[ri];
          if (logw) logw[k] = cw[ri];
        }
      }
      __syncthreads();
      continue;
    }
    // (d) children: runs of 8, kept in registers until all parents are read
    float nx[MAXR][RUN][DX];
    float nw[MAXR][RUN];
#pragma unroll
    for (int ri = 0; ri < MAXR; ++ri) {
      const int ka = RUN * (threadIdx.x + ri * TPB);
      if (ka < J) {
        int l = find_parent(st, J, ka);
#pragma unroll
        for (int g = 0; g < RUN / 4; ++g) {
          const int k0 = ka + 4 * g;
          if (k0 >= J) break;
          float z[4 * M::NZ];
          if (!last) group_noise<M::NZ, INJ>(a, f, t + 2, k0, z);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int k = k0 + e;
            if (k >= J) break;
            int adv = 0;
            while (l + 1 < J && st[l + 1] <= k) {
              ++l;
              if (++adv > 8) { l = find_parent(st, J, k); break; }
            }
            if (anc) anc[k] = l;
            float x[DX];
#pragma unroll
            for (int d = 0; d < DX; ++d) x[d] = xs[d * J + l];
            const float wb = rs ? base : ws[l];
            nw[ri][4 * g + e] = last ? 0.0f : wb + step1<M>(cr, ob, x, z + e * M::NZ);
#pragma unroll
            for (int d = 0; d < DX; ++d) nx[ri][4 * g + e][d] = x[d];
          }
        }
      }
    }
    __syncthreads();
    if (last) break;
#pragma unroll
    for (int ri = 0; ri < MAXR; ++ri) {
      const int ka = RUN * (threadIdx.x + ri * TPB);
#pragma unroll
      for (int e = 0; e < RUN; ++e) {
        const int k = ka + e;
        if (k < J) {
#pragma unroll
          for (int d = 0; d < DX; ++d) xs[d * J + k] = nx[ri][e][d];
          ws[k] = nw[ri][e];
          if (logw) logw[k] = nw[ri][e];
        }
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
  for (int d = 0; d < kMaxDim; ++d) { acc->fx[d] = 0.0; acc->px[d] = 0.0; }
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
      float z[M::NZ0 > 0 ? M::NZ0 : 1];
      step_noise<M>(a, f, j, 0, M::NZ0, z);
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
  const Acc& acc = *a.acc[p];
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
  const Acc& acc = *a.acc[p];
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


template <class M, int TPB, int IT, bool INJ>
int run_stream_t(Args& a, cudaStream_t s) {
  constexpr int TILE = TPB * IT;
  if (a.tile != TILE || a.ntiles != (a.J + TILE - 1) / TILE) return PPF_EINTERNAL;
  const size_t smem = sizeof(float) * M::MAXDX * TILE + sizeof(int) * (TILE + 4) + sizeof(float) * TILE;
  if (cudaFuncSetAttribute(k_resprop<M, TPB, IT, INJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return PPF_ECUDA;
  dim3 grid(a.ntiles, a.F);
  k_prep<M><<<(a.F + 127) / 128, 128, 0, s>>>(a);
  PROF_BEGIN(KIND_INIT);
  k_init<M, TPB, INJ><<<grid, TPB, 0, s>>>(a);
  PROF_END(KIND_INIT);
  for (int t = 0; t < a.T; ++t) {
    PROF_BEGIN(KIND_SUM);
    k_sum<M, TPB, IT><<<a.ntiles * a.F, TPB, 0, s>>>(a, t);
    PROF_END(KIND_SUM);
    PROF_BEGIN(KIND_RESPROP);
    k_resprop<M, TPB, IT, INJ><<<grid, TPB, smem, s>>>(a, t);
    PROF_END(KIND_RESPROP);
  }
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M, bool INJ>
int run_stream_tiled(Args& a, cudaStream_t s) {
  switch (a.tile) {
    case kTileLarge: return run_stream_t<M, 256, 8, INJ>(a, s);
    case kTileMid: return run_stream_t<M, 128, 4, INJ>(a, s);
    case kTileSmall: return run_stream_t<M, 64, 4, INJ>(a, s);
    default: return PPF_EINVAL;
  }
}

template <class M>
int run_stream(Args& a, cudaStream_t s) {
  if constexpr (M::WIDE) {
    // the wide LG (dx or dy above 4): exact arithmetic, Philox draws, the
    // 256-particle tiles (register-heavy particles, small CTAs)
    if (a.flags & PPF_F_INJECT) return PPF_EUNSUPPORTED;
    return a.tile == kTileSmall ? run_stream_t<M, 64, 4, false>(a, s) : PPF_EINTERNAL;
  } else {
    if ((a.flags & PPF_F_FAST) && !(a.flags & PPF_F_INJECT) && a.mode == MODE_PF) return run_stream_fast(a, s);
    return (a.flags & PPF_F_INJECT) ? run_stream_tiled<M, true>(a, s) : run_stream_tiled<M, false>(a, s);
  }
}

template <class M>
static int launch_prep(Args& a, cudaStream_t s) {
  k_prep<M><<<(a.F + 127) / 128, 128, 0, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

int run_prep(Args& a, cudaStream_t s) {
  switch (a.model.kind) {
        case PPF_MODEL_LG:
      return with_lg<int>(a.model, true, PPF_EUNSUPPORTED,
                          [&](auto tg) { return launch_prep<typename decltype(tg)::type>(a, s); });
    case PPF_MODEL_SV: return launch_prep<SV>(a, s);
    case PPF_MODEL_RICKER: return launch_prep<Ricker>(a, s);
    default: return PPF_EINVAL;
  }
}

template <class M>
size_t resident_smem(const Args& a) {
  return (size_t)a.J * sizeof(float) * (M::MAXDX + 1) + (size_t)(a.J + 4) * sizeof(int);
}

template <class M, int MAXR, bool INJ>
int launch_resident(Args& a, size_t smem, cudaStream_t s) {
  constexpr int TPB = 512;
  if (cudaFuncSetAttribute(k_resident<M, TPB, MAXR, INJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return PPF_ECUDA;
  PROF_BEGIN(KIND_RESIDENT);
  k_resident<M, TPB, MAXR, INJ><<<a.F, TPB, smem, s>>>(a);
  PROF_END(KIND_RESIDENT);
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M, bool INJ>
int run_resident_t(Args& a, cudaStream_t s) {
  constexpr int TPB = 512, RUN = 8;
  const size_t smem = resident_smem<M>(a);
  const int runs = (a.J + RUN * TPB - 1) / (RUN * TPB);   // runs of 8 children per thread
  if (smem > kResidentSmemMax || runs > 4) return PPF_EUNSUPPORTED;
  if (runs <= 1) return launch_resident<M, 1, INJ>(a, smem, s);
  if (runs <= 2) return launch_resident<M, 2, INJ>(a, smem, s);
  return launch_resident<M, 4, INJ>(a, smem, s);
}

template <class M>
int run_resident(Args& a, cudaStream_t s) {
  return (a.flags & PPF_F_INJECT) ? run_resident_t<M, true>(a, s) : run_resident_t<M, false>(a, s);
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
    case PPF_PATH_RESIDENT:
      if constexpr (M::WIDE) return PPF_EUNSUPPORTED;   // the wide LG streams only
      else return run_resident<M>(a, s);
    default: return PPF_EINVAL;
  }
}

int run_pfilter_path(Args& a, int path, cudaStream_t s) {
  if (path == PPF_PATH_CLUSTER) return run_cluster(a, false, s);
  switch (a.model.kind) {
        case PPF_MODEL_LG:
      return with_lg<int>(a.model, true, PPF_EUNSUPPORTED,
                          [&](auto tg) { return dispatch_model<typename decltype(tg)::type>(a, path, s); });
    case PPF_MODEL_SV: return dispatch_model<SV>(a, path, s);
    case PPF_MODEL_RICKER: return dispatch_model<Ricker>(a, path, s);
    default: return PPF_EINVAL;
  }
}

int run_stream_any(Args& a, cudaStream_t s) { return run_pfilter_path(a, PPF_PATH_STREAM, s); }

size_t resident_smem_bytes(const Args& a) {
  return (size_t)a.J * sizeof(float) * (a.model.dx + 1) + (size_t)(a.J + 4) * sizeof(int);
}

}  // namespace ppf
