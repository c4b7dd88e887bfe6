// ppf_fast.cu -- the streaming batched particle filter with PPF_F_FAST.
//
// The same kernels as the streaming path of ppf_pfilter.cu (the tile bodies
// of ppf_stream.cuh and ppf_kernels.cuh), instantiated with FAST = true:
//  - Box-Muller normals from the same Philox4x32-10 words through the SFU
//    approximations (pp_boxmuller_fast: __log2f, rsqrtf, __sincosf);
//  - the resampling weights' exponential e = exp(w - max) through __expf;
//  - this file is compiled with floating-point contraction (-fmad=true), so
//    the model arithmetic may fuse multiply-adds.
// Everything else is unchanged: the exact fixed-point CDF and systematic
// offsets, the Philox counters, float64 log-likelihood terms.  The results
// are therefore not bit-identical with the C oracle, only statistically
// equivalent; the kernels here have their own names, so no instantiation is
// shared with the exact translation units.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ppf.h"
#include "ppf_core.cuh"
#include "ppf_internal.h"
#include "ppf_kernels.cuh"
#include "ppf_models.cuh"
#include "ppf_stream.cuh"

namespace ppf {

template <class M, int TPB>
__global__ void __launch_bounds__(TPB) k_init_fast(Args a) {
  init_tile<M, TPB, false, true>(a, blockIdx.y, blockIdx.x);
}

template <class M, int TPB, int IT>
__global__ void __launch_bounds__(TPB) k_sum_fast(Args a, int t) {
  const int v = blockIdx.x;
  sum_tile<M, TPB, IT, true, true>(a, t, v / a.ntiles, v % a.ntiles);
}

template <class M, int TPB, int IT>
__global__ void __launch_bounds__(TPB, RespropOccupancy<M>::B * (256 / TPB)) k_resprop_fast(Args a, int t) {
  resprop_tile<M, TPB, IT, false, true, true>(a, t, blockIdx.y, blockIdx.x);
}

template <class M, int TPB, int IT>
static int run_fast_t(Args& a, cudaStream_t s) {
  constexpr int TILE = TPB * IT;
  if (a.tile != TILE || a.ntiles != (a.J + TILE - 1) / TILE) return PPF_EINTERNAL;
  const size_t smem = sizeof(float) * M::MAXDX * TILE + sizeof(int) * (TILE + 4) + sizeof(float) * TILE;
  if (cudaFuncSetAttribute(k_resprop_fast<M, TPB, IT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return PPF_ECUDA;
  dim3 grid(a.ntiles, a.F);
  const int rc = run_prep(a, s);
  if (rc) return rc;
  PROF_BEGIN(KIND_INIT);
  k_init_fast<M, TPB><<<grid, TPB, 0, s>>>(a);
  PROF_END(KIND_INIT);
  for (int t = 0; t < a.T; ++t) {
    PROF_BEGIN(KIND_SUM);
    k_sum_fast<M, TPB, IT><<<a.ntiles * a.F, TPB, 0, s>>>(a, t);
    PROF_END(KIND_SUM);
    PROF_BEGIN(KIND_RESPROP);
    k_resprop_fast<M, TPB, IT><<<grid, TPB, smem, s>>>(a, t);
    PROF_END(KIND_RESPROP);
  }
  return cudaGetLastError() == cudaSuccess ? PPF_OK : PPF_ECUDA;
}

template <class M>
static int run_fast_m(Args& a, cudaStream_t s) {
  switch (a.tile) {
    case kTileLarge: return run_fast_t<M, 256, 8>(a, s);
    case kTileMid: return run_fast_t<M, 128, 4>(a, s);
    case kTileSmall: return run_fast_t<M, 64, 4>(a, s);
    default: return PPF_EINVAL;
  }
}

int run_stream_fast(Args& a, cudaStream_t s) {
  switch (a.model.kind) {
        case PPF_MODEL_LG:
      return with_lg<int>(a.model, false, PPF_EUNSUPPORTED,
                          [&](auto tg) { return run_fast_m<typename decltype(tg)::type>(a, s); });
    case PPF_MODEL_SV: return run_fast_m<SV>(a, s);
    case PPF_MODEL_RICKER: return run_fast_m<Ricker>(a, s);
    default: return PPF_EINVAL;
  }
}

}  // namespace ppf
