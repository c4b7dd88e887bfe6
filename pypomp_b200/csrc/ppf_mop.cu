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
// children read the stored offsets, so they are deterministic.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "ppf.h"
#include "ppf_core.cuh"
#include "ppf_internal.h"
#include "ppf_kernels.cuh"
#include "ppf_models.cuh"

namespace ppf {

constexpr int kMaxNG = 64;

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
    for (int k = lo; k < hi; ++k) {
#pragma unroll
      for (int d = 0; d < DX; ++d) lx[d] += lxi[d * J + k];
      lw += lwi[k];
    }
    const float gl = -1.0f;                       // d(-sum ll)/d ll_t
    const float lm = lw + gl * pi;
    const float lwP = lw + gl * (pi - 1.0f / (float)J);
    if (m == m && m > -INFINITY) M::bwd(cr, x, z, kp, lm, lx, g);
    else {
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

template <int DX, int DYS>
struct Chain<LG<DX, DYS>> {
  __device__ static double map(const ppf_model& m, const float* th, const double* gn, int p, bool est) {
    const int dy = m.dy;
    const int nA = DX * DX, nC = dy * DX, nQ = DX * (DX + 1) / 2, nR = dy * (dy + 1) / 2;
    if (p < nA) return gn[LG<DX, DYS>::GA + p];
    p -= nA;
    if (p < nC) return gn[LG<DX, DYS>::GC + p];
    p -= nC;
    if (p < nQ) {
      double v = gn[LG<DX, DYS>::GQ + p];
      for (int i = 0; i < DX; ++i)
        if (est && p == i * (i + 1) / 2 + i) v *= (double)pp_expf(th[nA + nC + p]);
      return v;
    }
    p -= nQ;
    if (p < nR) {
      double v = gn[LG<DX, DYS>::GR + p];
      for (int i = 0; i < dy; ++i)
        if (est && p == i * (i + 1) / 2 + i) v *= (double)pp_expf(th[nA + nC + nQ + p]);
      return v;
    }
    p -= nR;
    return gn[LG<DX, DYS>::GX0 + p];
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
// host orchestration
// ---------------------------------------------------------------------------

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
int run_mop_model(Args& a, const MopWork& w, cudaStream_t s) {
  int rc = run_stream_any(a, s);
  if (rc || !w.grad) return rc;
  return (a.flags & PPF_F_INJECT) ? mop_backward<M, true>(a, w, s) : mop_backward<M, false>(a, w, s);
}

int run_mop(Args& a, const MopWork& w, cudaStream_t s) {
  switch (a.model.kind) {
    case PPF_MODEL_LG:
      switch (a.model.dx) {
        case 1: return a.model.dy == 1 ? run_mop_model<LG<1, 1>>(a, w, s) : run_mop_model<LG<1>>(a, w, s);
        case 2: return a.model.dy == 2 ? run_mop_model<LG<2, 2>>(a, w, s) : run_mop_model<LG<2>>(a, w, s);
        case 3: return a.model.dy == 3 ? run_mop_model<LG<3, 3>>(a, w, s) : run_mop_model<LG<3>>(a, w, s);
        case 4: return a.model.dy == 4 ? run_mop_model<LG<4, 4>>(a, w, s) : run_mop_model<LG<4>>(a, w, s);
        default: return PPF_EUNSUPPORTED;
      }
    case PPF_MODEL_SV: return run_mop_model<SV>(a, w, s);
    case PPF_MODEL_RICKER: return run_mop_model<Ricker>(a, w, s);
    default: return PPF_EINVAL;
  }
}

template <class M>
int run_mop_backward_model(Args& a, const MopWork& w, cudaStream_t s) {
  return (a.flags & PPF_F_INJECT) ? mop_backward<M, true>(a, w, s) : mop_backward<M, false>(a, w, s);
}

int run_mop_backward(Args& a, const MopWork& w, cudaStream_t s) {
  switch (a.model.kind) {
    case PPF_MODEL_LG:
      switch (a.model.dx) {
        case 1: return a.model.dy == 1 ? run_mop_backward_model<LG<1, 1>>(a, w, s) : run_mop_backward_model<LG<1>>(a, w, s);
        case 2: return a.model.dy == 2 ? run_mop_backward_model<LG<2, 2>>(a, w, s) : run_mop_backward_model<LG<2>>(a, w, s);
        case 3: return a.model.dy == 3 ? run_mop_backward_model<LG<3, 3>>(a, w, s) : run_mop_backward_model<LG<3>>(a, w, s);
        case 4: return a.model.dy == 4 ? run_mop_backward_model<LG<4, 4>>(a, w, s) : run_mop_backward_model<LG<4>>(a, w, s);
        default: return PPF_EUNSUPPORTED;
      }
    case PPF_MODEL_SV: return run_mop_backward_model<SV>(a, w, s);
    case PPF_MODEL_RICKER: return run_mop_backward_model<Ricker>(a, w, s);
    default: return PPF_EINVAL;
  }
}

}  // namespace ppf
