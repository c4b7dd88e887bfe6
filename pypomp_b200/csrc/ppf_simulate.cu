// ppf_simulate.cu -- trajectories of the built-in models: rinit, then rproc
// and rmeas for each observation time (pypomp/core/algorithms/simulate.py:15-142,
// _simulate_internal / _simulate_helper), one thread per (parameter set,
// replicate).
//
// Each thread keeps its state in registers.  The trajectory is staged in
// shared memory kSimChunk time points at a time; the CTA then writes the
// staged rows out in the reference's layout, X[F][nsim][T+1][dx] and
// Y[F][nsim][T][dy], with consecutive threads on consecutive addresses of
// one replicate's rows.  Per trajectory step the kernel writes (dx + dy)
// floats: HBM-bound on writes when the draws are cheap, issue-bound on the
// Philox / Box-Muller / Poisson arithmetic otherwise.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ppf.h"
#include "ppf_internal.h"
#include "ppf_models.cuh"
#include "ppf_philox.h"
#include "ppf_sample.h"

namespace ppf {

constexpr int kSimTPB = 128;
constexpr int kSimChunk = 8;

struct SimArgs {
  ppf_model model;
  int F, nsim, T;
  bool est;
  const float* theta;
  const uint64_t* seeds;
  float* X;
  float* Y;
};

// Copy nlive staged rows of L floats (shared row stride sstride) to global rows
// of stride gstride.  A warp covers 32 / L rows per pass when L <= 32, so each
// lane finds its row and offset once per flush rather than per element.
__device__ __forceinline__ void flush_rows(float* g, size_t gstride, const float* sm, int sstride, int L,
                                           int nlive) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = kSimTPB / 32;
  if (L <= 32) {
    const int rpi = 32 / L;
    const int rr = lane / L, o = lane - rr * L;
    if (rr < rpi)
      for (int r = warp * rpi + rr; r < nlive; r += NW * rpi) g[(size_t)r * gstride + o] = sm[r * sstride + o];
  } else {
    for (int r = warp; r < nlive; r += NW)
      for (int o = lane; o < L; o += 32) g[(size_t)r * gstride + o] = sm[r * sstride + o];
  }
}

template <class M>
__global__ void __launch_bounds__(kSimTPB) k_simulate(SimArgs s) {
  constexpr int DX = M::MAXDX, DYM = M::MAXDY;
  // time points staged per flush: fewer for the wide LG, whose rows are long
  constexpr int CH = M::WIDE ? 2 : kSimChunk;
  constexpr int XS = CH * DX + 1, YS = CH * DYM + 1;   // odd row strides
  __shared__ typename M::Consts cs;
  __shared__ float xs[kSimTPB * XS];
  __shared__ float ys[kSimTPB * YS];
  const int f = blockIdx.y;
  const int kb = blockIdx.x * kSimTPB;
  const int k = kb + threadIdx.x;
  const int nlive = min(kSimTPB, s.nsim - kb);
  const bool live = k < s.nsim;
  const int P = s.model.n_params, dy = s.model.dy;
  if (threadIdx.x == 0) M::prepare(cs, s.theta + (size_t)f * P, s.model, s.est);
  __syncthreads();
  const typename M::Consts& c = cs;
  const uint64_t seed = s.seeds[f];
  float* Xf = s.X + ((size_t)f * s.nsim + kb) * (size_t)(s.T + 1) * DX;
  float* Yf = s.Y + ((size_t)f * s.nsim + kb) * (size_t)s.T * dy;

  float x[DX];
  int tb = 0;   // first time point of the staged chunk (0 = the initial state)
  for (int tau = 0; tau <= s.T; ++tau) {
    const int slot = tau - tb;
    if (live) {
      if (tau == 0) {
        float z0[M::NZ0 > 0 ? M::NZ0 : 1];
        if (M::NZ0 > 0) pp_normals_own(seed, (uint32_t)k, 0u, PPF_TAG_PROCESS, M::NZ0, z0);
        M::rinit(c, z0, x);
      } else {
        float z[M::NZ];
        pp_normals_own(seed, (uint32_t)k, (uint32_t)tau, PPF_TAG_PROCESS, M::NZ, z);
        M::rproc(c, x, z);
        float y[DYM];
        M::rmeas(c, x, seed, (uint32_t)k, (uint32_t)tau, y);
#pragma unroll
        for (int i = 0; i < DYM; ++i)
          if (i < dy) ys[threadIdx.x * YS + slot * dy + i] = y[i];
      }
#pragma unroll
      for (int d = 0; d < DX; ++d) xs[threadIdx.x * XS + slot * DX + d] = x[d];
    }
    if (slot == CH - 1 || tau == s.T) {
      __syncthreads();
      // states of time points tb..tau, one contiguous run per replicate
      flush_rows(Xf + (size_t)tb * DX, (size_t)(s.T + 1) * DX, xs, XS, (tau - tb + 1) * DX, nlive);
      // observations of time points max(tb, 1)..tau, i.e. y indices from max(tb, 1) - 1
      const int t0 = tb > 0 ? tb : 1;
      if (tau >= t0)
        flush_rows(Yf + (size_t)(t0 - 1) * dy, (size_t)s.T * dy, ys + (t0 - tb) * dy, YS, (tau - t0 + 1) * dy,
                   nlive);
      __syncthreads();
      tb = tau + 1;
    }
  }
}

template <class M>
static int launch_simulate(const SimArgs& a, cudaStream_t s) {
  const dim3 grid((a.nsim + kSimTPB - 1) / kSimTPB, a.F, 1);
  PROF_BEGIN(KIND_SIMULATE);
  k_simulate<M><<<grid, kSimTPB, 0, s>>>(a);
  PROF_END(KIND_SIMULATE);
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

int run_simulate(const ppf_simulate_desc* d, cudaStream_t st) {
  SimArgs s;
  s.model = d->model;
  s.F = d->F;
  s.nsim = d->nsim;
  s.T = d->T;
  s.est = (d->flags & PPF_F_EST) != 0;
  s.theta = d->theta;
  s.seeds = d->seeds;
  s.X = d->X;
  s.Y = d->Y;
  switch (d->model.kind) {
        case PPF_MODEL_LG:
      return with_lg<int>(d->model, true, PPF_EINVAL,
                          [&](auto tg) { return launch_simulate<typename decltype(tg)::type>(s, st); });
    case PPF_MODEL_SV: return launch_simulate<SV>(s, st);
    case PPF_MODEL_RICKER: return launch_simulate<Ricker>(s, st);
    default: return PPF_EINVAL;
  }
}

}  // namespace ppf
