// ppf_models.cuh -- device code of the built-in models (LG, SV, Ricker).
//
// Each model is a struct with a per-filter constant block (`Consts`, kept in
// shared memory by the kernels) and the three mechanics the reference's
// plugin boundary calls per particle (pypomp/functional/structs.py:10-75):
//   rinit  -- pypomp/models/linear_gaussian.py:139 (_rinit)
//   rproc  -- linear_gaussian.py:151 (_rproc), one Euler step (nstep = 1)
//   dmeas  -- linear_gaussian.py:166 (_dmeas)
// plus rmeas (linear_gaussian.py:180-191, _rmeas) for simulation, drawing its
// noise from the measurement streams of ppf_sample.h.
// The operation order below is the arithmetic definition that the C oracle
// (oracle/ppf_oracle.c) restates; float32 throughout, elementary functions
// from ppf_detmath.h, compiled with -fmad=false so no contraction happens.
#pragma once

#include <stdint.h>
#include "ppf.h"
#include "ppf_detmath.h"
#include "ppf_sample.h"

#define PPF_LOG2PI_F 1.83787706640934548356f

namespace ppf {

// ---------------------------------------------------------------------------
// Linear Gaussian (dx, dy <= 9, pypomp/models/linear_gaussian.py:48 MAX_DIM).
// Parameter order as LG's canonical names: A (row-major dx*dx), C (row-major
// dy*dx), lower triangle of chol(Q) row-major, lower triangle of chol(R)
// row-major, X0 (dx).
// ---------------------------------------------------------------------------
// DYS > 0 fixes the observation dimension at compile time (the dispatch uses
// it for dy == dx <= 4): the measurement loops become static and the model
// constants stay in registers.  DYS == 0 reads dy (<= MDY) at run time.  The
// matrices are stored with row stride S: 4 for the models up to 4 x 4, 9 for
// the wide ones (dx or dy above 4), whose constant block is 2 KB.
template <int DX, int DYS = 0, int MDY = 4>
struct LG {
  static constexpr int kind = PPF_MODEL_LG;
  static constexpr int MAXDX = DX;     // state dimension, fixed per instantiation
  static constexpr int NZ = DX;        // process normals per particle-step
  static constexpr int NZ0 = DX;       // initial-state normals per particle
  static constexpr int MAXDY = DYS > 0 ? DYS : MDY;
  static constexpr bool WIDE = (DX > 4 || MAXDY > 4);
  static constexpr int S = WIDE ? 9 : 4;                      // row stride of the matrices
  static constexpr int CONST_BYTES = WIDE ? 2048 : 512;       // workspace bytes per filter
  static constexpr int MAXP = DX * DX + MAXDY * DX + DX * (DX + 1) / 2 + MAXDY * (MAXDY + 1) / 2 + DX;
  struct Consts {
    int dx, dy;
    float A[S * S], C[S * S], LQ[S * S], L[S * S], Linv[S], X0[S];
    float c0;
    float LR[S * S];   // the parameter factor of R, as rmeas draws with it
  };
  __device__ static __forceinline__ int ndy(const Consts& c) { return DYS > 0 ? DYS : c.dy; }
  __device__ static void prepare(Consts& c, const float* th, const ppf_model& m, bool est) {
    const int dx = DX, dy = DYS > 0 ? DYS : m.dy;   // DYS, when set, equals m.dy (the dispatch checks)
    c.dx = dx; c.dy = dy;
    int p = 0;
    for (int i = 0; i < dx; ++i)
      for (int k = 0; k < dx; ++k) c.A[i * S + k] = th[p++];
    for (int i = 0; i < dy; ++i)
      for (int k = 0; k < dx; ++k) c.C[i * S + k] = th[p++];
    float* LR = c.LR;
    for (int i = 0; i < S * S; ++i) { c.LQ[i] = 0.0f; LR[i] = 0.0f; c.L[i] = 0.0f; }
    for (int i = 0; i < dx; ++i)
      for (int k = 0; k <= i; ++k) {
        float v = th[p++];
        if (est && i == k) v = pp_expf(v);
        c.LQ[i * S + k] = v;
      }
    for (int i = 0; i < dy; ++i)
      for (int k = 0; k <= i; ++k) {
        float v = th[p++];
        if (est && i == k) v = pp_expf(v);
        LR[i * S + k] = v;
      }
    for (int i = 0; i < dx; ++i) c.X0[i] = th[p++];
    // R = LR LR^T, then its Cholesky factor (as multivariate_normal.logpdf does).
    float R[S * S];
    for (int i = 0; i < dy; ++i)
      for (int k = 0; k <= i; ++k) {
        float s = 0.0f;
        for (int l = 0; l <= k; ++l) s = s + LR[i * S + l] * LR[k * S + l];
        R[i * S + k] = s;
      }
    for (int i = 0; i < dy; ++i)
      for (int k = 0; k <= i; ++k) {
        float s = R[i * S + k];
        for (int l = 0; l < k; ++l) s = s - c.L[i * S + l] * c.L[k * S + l];
        if (i == k) c.L[i * S + i] = sqrtf(s);
        else c.L[i * S + k] = s / c.L[k * S + k];
      }
    float c0 = -0.5f * (float)dy * PPF_LOG2PI_F;
    for (int i = 0; i < dy; ++i) {
      c.Linv[i] = 1.0f / c.L[i * S + i];
      c0 = c0 - pp_logf(c.L[i * S + i]);
    }
    c.c0 = c0;
  }

  __device__ static void rinit(const Consts& c, const float* z, float* x) {
#pragma unroll
    for (int i = 0; i < DX; ++i) {
      float acc = c.X0[i];
#pragma unroll
      for (int k = 0; k <= i; ++k) acc = pp_fma(c.LQ[i * S + k], z[k], acc);
      x[i] = acc;
    }
  }

  __device__ static void rproc(const Consts& c, float* x, const float* z) {
    float y[DX];
#pragma unroll
    for (int i = 0; i < DX; ++i) {
      float acc = 0.0f;
#pragma unroll
      for (int k = 0; k < DX; ++k) acc = pp_fma(c.A[i * S + k], x[k], acc);
#pragma unroll
      for (int k = 0; k <= i; ++k) acc = pp_fma(c.LQ[i * S + k], z[k], acc);
      y[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < DX; ++i) x[i] = y[i];
  }

  __device__ static float dmeas(const Consts& c, const float* y, float /*ycon*/, const float* x) {
    float s[MAXDY];
    float q = 0.0f;
#pragma unroll
    for (int i = 0; i < MAXDY; ++i) {
      if (i < ndy(c)) {
        float a = 0.0f;
#pragma unroll
        for (int k = 0; k < DX; ++k) a = pp_fma(c.C[i * S + k], x[k], a);
        float r = y[i] - a;
#pragma unroll
        for (int l = 0; l < i; ++l) r = pp_fma(-c.L[i * S + l], s[l], r);
        s[i] = r * c.Linv[i];
        q = pp_fma(s[i], s[i], q);
      }
    }
    return pp_fma(-0.5f, q, c.c0);
  }

  // y = C x + L_R w, w ~ N(0, I_dy).  MEAS_NZ: measurement normals per draw
  // when fixed at compile time (0: dy known only at run time).
  static constexpr int MEAS_NZ = DYS;
  __device__ static void rmeas_z(const Consts& c, const float* x, const float* w, float* y) {
#pragma unroll
    for (int i = 0; i < MAXDY; ++i) {
      if (i < ndy(c)) {
        float a = 0.0f;
#pragma unroll
        for (int q = 0; q < DX; ++q) a = pp_fma(c.C[i * S + q], x[q], a);
#pragma unroll
        for (int l = 0; l <= i; ++l) a = pp_fma(c.LR[i * S + l], w[l], a);
        y[i] = a;
      }
    }
  }
  __device__ static void rmeas(const Consts& c, const float* x, uint64_t seed, uint32_t k, uint32_t s,
                               float* y) {
    float w[MAXDY];
    pp_normals_own(seed, k, s, PPF_TAG_MEASURE, ndy(c), w);
    rmeas_z(c, x, w, y);
  }

  // ---- adjoint (MOP-alpha gradient).  Natural-scale gradient in a padded
  // layout with static indices: A[DX*DX] | C[MAXDY*DX] | LQ tril(DX) |
  // LR tril(MAXDY) | X0[DX]; the host maps it to the canonical order.
  static constexpr int NQ = DX * (DX + 1) / 2;
  static constexpr int GA = 0, GC = DX * DX, GQ = GC + MAXDY * DX, GR = GQ + NQ,
                       GX0 = GR + MAXDY * (MAXDY + 1) / 2;
  static constexpr int NG = GX0 + DX;
  struct Keep {
    float xP[DX];
    float s[MAXDY];
  };
  __device__ static float fwd_keep(const Consts& c, const float* y, float, const float* xin,
                                   const float* z, Keep& k) {
#pragma unroll
    for (int i = 0; i < DX; ++i) k.xP[i] = xin[i];
    rproc(c, k.xP, z);
    float q = 0.0f;
#pragma unroll
    for (int i = 0; i < MAXDY; ++i) {
      k.s[i] = 0.0f;
      if (i < ndy(c)) {
        float a = 0.0f;
#pragma unroll
        for (int kk = 0; kk < DX; ++kk) a = pp_fma(c.C[i * S + kk], k.xP[kk], a);
        float r = y[i] - a;
#pragma unroll
        for (int l = 0; l < i; ++l) r = pp_fma(-c.L[i * S + l], k.s[l], r);
        k.s[i] = r * c.Linv[i];
        q = pp_fma(k.s[i], k.s[i], q);
      }
    }
    return pp_fma(-0.5f, q, c.c0);
  }
  // lx: in = adjoint of x^P from the children, out = adjoint of xin.
  __device__ static void bwd(const Consts& c, const float* xin, const float* z, const Keep& k,
                             float lm, float* lx, float* g) {
    // v = L^-T s
    float v[MAXDY];
#pragma unroll
    for (int i = MAXDY - 1; i >= 0; --i) {
      v[i] = 0.0f;
      if (i < ndy(c)) {
        float r = k.s[i];
#pragma unroll
        for (int l = i + 1; l < MAXDY; ++l)
          if (l < ndy(c)) r = r - c.L[l * S + i] * v[l];
        v[i] = r * c.Linv[i];
      }
    }
    float lxP[DX];
#pragma unroll
    for (int kk = 0; kk < DX; ++kk) {
      float a = lx[kk];
#pragma unroll
      for (int i = 0; i < MAXDY; ++i)
        if (i < ndy(c)) a = a + lm * c.C[i * S + kk] * v[i];
      lxP[kk] = a;
    }
#pragma unroll
    for (int i = 0; i < MAXDY; ++i)
      if (i < ndy(c)) {
#pragma unroll
        for (int kk = 0; kk < DX; ++kk) g[GC + i * DX + kk] += lm * v[i] * k.xP[kk];
#pragma unroll
        for (int l = 0; l <= i; ++l) g[GR + i * (i + 1) / 2 + l] += lm * v[i] * k.s[l];
        g[GR + i * (i + 1) / 2 + i] -= lm * c.Linv[i];
      }
#pragma unroll
    for (int i = 0; i < DX; ++i) {
#pragma unroll
      for (int kk = 0; kk < DX; ++kk) g[GA + i * DX + kk] += lxP[i] * xin[kk];
#pragma unroll
      for (int kk = 0; kk <= i; ++kk) g[GQ + i * (i + 1) / 2 + kk] += lxP[i] * z[kk];
    }
#pragma unroll
    for (int kk = 0; kk < DX; ++kk) {
      float a = 0.0f;
#pragma unroll
      for (int i = 0; i < DX; ++i) a = a + c.A[i * S + kk] * lxP[i];
      lx[kk] = a;
    }
  }
  __device__ static void bwd_init(const Consts&, const float* z0, const float* lx0, float* g) {
#pragma unroll
    for (int i = 0; i < DX; ++i) {
      g[GX0 + i] += lx0[i];
#pragma unroll
      for (int kk = 0; kk <= i; ++kk) g[GQ + i * (i + 1) / 2 + kk] += lx0[i] * z0[kk];
    }
  }
};

// ---------------------------------------------------------------------------
// Heston-type log-variance stochastic volatility.  State (v, eps); parameters
// (kappa, theta, xi, rho, mu, v0); estimation scale log/log/log/atanh/id/id.
//   v' = v + kappa (theta - e^v) e^-v dt + xi e^{-v/2} sqrt(dt) eps'
//   r  ~ N(mu dt + rho sqrt(e^{v'} dt) eps', (1 - rho^2) e^{v'} dt)
// ---------------------------------------------------------------------------
__host__ __device__ inline float pp_tanhf_det(float a) {
  const float e = pp_expf(-2.0f * fabsf(a));
  const float t = (1.0f - e) / (1.0f + e);
  return a < 0.0f ? -t : t;
}

struct SV {
  static constexpr int kind = PPF_MODEL_SV;
  static constexpr int MAXDX = 2;
  static constexpr int NZ = 1;
  static constexpr int NZ0 = 0;
  static constexpr int MAXDY = 1;
  static constexpr bool WIDE = false;
  static constexpr int CONST_BYTES = 512;
  static constexpr int MAXP = 6;
  struct Consts {
    int dx, dy;
    float kappa, theta, xi, rho, mu, v0, dt, sqdt, mudt, rhoc, c0, kdt, xsq;
  };

  __device__ static void prepare(Consts& c, const float* th, const ppf_model& m, bool est) {
    c.dx = 2; c.dy = 1;
    c.kappa = est ? pp_expf(th[0]) : th[0];
    c.theta = est ? pp_expf(th[1]) : th[1];
    c.xi = est ? pp_expf(th[2]) : th[2];
    c.rho = est ? pp_tanhf_det(th[3]) : th[3];
    c.mu = th[4];
    c.v0 = th[5];
    c.dt = m.dt;
    c.sqdt = sqrtf(m.dt);
    c.mudt = c.mu * c.dt;
    c.rhoc = sqrtf(1.0f - c.rho * c.rho);
    c.c0 = -0.5f * PPF_LOG2PI_F - pp_logf(c.rhoc) - 0.5f * pp_logf(c.dt);
    c.kdt = c.kappa * c.dt;
    c.xsq = c.xi * c.sqdt;
  }
  __device__ static void rinit(const Consts& c, const float*, float* x) {
    x[0] = c.v0;
    x[1] = 0.0f;
  }
  // (theta - e^v) e^-v = theta e^-v - 1;  e^-v = (e^{-v/2})^2
  __device__ static void rproc(const Consts& c, float* x, const float* z) {
    const float v = x[0];
    const float emh = pp_expf(-0.5f * v);
    const float emv = emh * emh;
    const float a1 = pp_fma(c.theta, emv, -1.0f);
    const float v1 = pp_fma(c.kdt, a1, v);
    x[0] = pp_fma(c.xsq * emh, z[0], v1);
    x[1] = z[0];
  }
  __device__ static float dmeas(const Consts& c, const float* y, float, const float* x) {
    const float v = x[0];
    const float sd = pp_expf(0.5f * v) * c.sqdt;
    const float mean = pp_fma(c.rho * sd, x[1], c.mudt);
    const float r = (y[0] - mean) / (c.rhoc * sd);
    return pp_fma(-0.5f * r, r, pp_fma(-0.5f, v, c.c0));
  }
  // r = mu dt + rho sd eps + sqrt(1 - rho^2) sd w,  sd = e^{v/2} sqrt(dt)
  static constexpr int MEAS_NZ = 1;
  __device__ static void rmeas_z(const Consts& c, const float* x, const float* w, float* y) {
    const float sd = pp_expf(0.5f * x[0]) * c.sqdt;
    const float mean = pp_fma(c.rho * sd, x[1], c.mudt);
    y[0] = pp_fma(c.rhoc * sd, w[0], mean);
  }
  __device__ static void rmeas(const Consts& c, const float* x, uint64_t seed, uint32_t k, uint32_t s,
                               float* y) {
    float w[1];
    pp_normals_own(seed, k, s, PPF_TAG_MEASURE, 1, w);
    rmeas_z(c, x, w, y);
  }

  // ---- adjoint: natural-scale gradient in canonical order
  // (kappa, theta, xi, rho, mu, v0).
  static constexpr int NG = 6;
  struct Keep {
    float xP[2];
    float emh, sd, r, A;
  };
  __device__ static float fwd_keep(const Consts& c, const float* y, float, const float* xin,
                                   const float* z, Keep& k) {
    k.xP[0] = xin[0];
    k.xP[1] = xin[1];
    k.emh = pp_expf(-0.5f * xin[0]);
    rproc(c, k.xP, z);
    const float v = k.xP[0];
    k.sd = pp_expf(0.5f * v) * c.sqdt;
    const float mean = pp_fma(c.rho * k.sd, k.xP[1], c.mudt);
    k.r = (y[0] - mean) / (c.rhoc * k.sd);
    k.A = (y[0] - c.mudt) / k.sd;
    return pp_fma(-0.5f * k.r, k.r, pp_fma(-0.5f, v, c.c0));
  }
  __device__ static void bwd(const Consts& c, const float* xin, const float* z, const Keep& k,
                             float lm, float* lx, float* g) {
    const float rc = c.rhoc;
    const float eps = k.xP[1];
    // dmeas: d/dv' = r A/(2 rc) - 1/2 ; d/deps = r rho / rc
    const float dgv = 0.5f * k.r * k.A / rc - 0.5f;
    const float dge = k.r * c.rho / rc;
    const float rc3 = rc * rc * rc;
    g[3] += lm * (-k.r * (k.A * c.rho - eps) / rc3 + c.rho / (rc * rc));
    g[4] += lm * (k.r * c.dt / (rc * k.sd));
    const float lv = lx[0] + lm * dgv;          // adjoint of v'
    // (eps' = z has no parameter or state dependence; its adjoint lx[1] + lm dge stops here)
    (void)dge;
    // rproc: v' = v + kappa dt (theta e^-v - 1) + xi sqrt(dt) e^{-v/2} z
    const float emv = k.emh * k.emh;
    g[0] += lv * c.dt * (c.theta * emv - 1.0f);
    g[1] += lv * c.kappa * c.dt * emv;
    g[2] += lv * c.sqdt * k.emh * z[0];
    const float dvv = 1.0f - c.kdt * c.theta * emv - 0.5f * c.xsq * k.emh * z[0];
    lx[0] = lv * dvv;
    lx[1] = 0.0f;
    (void)xin;
  }
  __device__ static void bwd_init(const Consts&, const float*, const float* lx0, float* g) {
    g[5] += lx0[0];
  }
};

// ---------------------------------------------------------------------------
// Stochastic Ricker: N' = r N exp(-N + sigma e), y ~ Poisson(phi N').
// Parameters (r, sigma, phi, N_0); estimation scale log of each.
// ---------------------------------------------------------------------------
struct Ricker {
  static constexpr int kind = PPF_MODEL_RICKER;
  static constexpr int MAXDX = 1;
  static constexpr int NZ = 1;
  static constexpr int NZ0 = 0;
  static constexpr int MAXDY = 1;
  static constexpr bool WIDE = false;
  static constexpr int CONST_BYTES = 512;
  static constexpr int MAXP = 4;
  struct Consts {
    int dx, dy;
    float r, sigma, phi, N0;
  };

  __device__ static void prepare(Consts& c, const float* th, const ppf_model&, bool est) {
    c.dx = 1; c.dy = 1;
    c.r = est ? pp_expf(th[0]) : th[0];
    c.sigma = est ? pp_expf(th[1]) : th[1];
    c.phi = est ? pp_expf(th[2]) : th[2];
    c.N0 = est ? pp_expf(th[3]) : th[3];
  }
  __device__ static void rinit(const Consts& c, const float*, float* x) { x[0] = c.N0; }
  __device__ static void rproc(const Consts& c, float* x, const float* z) {
    const float N = x[0];
    x[0] = (c.r * N) * pp_expf(pp_fma(c.sigma, z[0], -N));
  }
  __device__ static float dmeas(const Consts& c, const float* y, float ycon, const float* x) {
    const float lam = c.phi * x[0];
    if (y[0] == 0.0f) return -lam;
    return pp_fma(y[0], pp_logf(lam), -lam) - ycon;
  }
  // y ~ Poisson(phi N): counts, no measurement normals
  static constexpr int MEAS_NZ = 0;
  __device__ static void rmeas_z(const Consts&, const float*, const float*, float*) {}
  __device__ static void rmeas(const Consts& c, const float* x, uint64_t seed, uint32_t k, uint32_t s,
                               float* y) {
    y[0] = pp_poisson(c.phi * x[0], seed, k, s);
  }

  // ---- adjoint: natural-scale gradient in canonical order (r, sigma, phi, N_0).
  static constexpr int NG = 4;
  struct Keep {
    float xP[1];
    float y;
  };
  __device__ static float fwd_keep(const Consts& c, const float* y, float ycon, const float* xin,
                                   const float* z, Keep& k) {
    k.xP[0] = xin[0];
    rproc(c, k.xP, z);
    k.y = y[0];
    return dmeas(c, y, ycon, k.xP);
  }
  __device__ static void bwd(const Consts& c, const float* xin, const float* z, const Keep& k,
                             float lm, float* lx, float* g) {
    const float Np = k.xP[0];
    const float N = xin[0];
    // dmeas: y log(phi N') - phi N' - log y!, d/dN' = y / N' - phi.  The
    // weight adjoint lm carries the particle's weight, which scales like
    // N'^y, so lm * y / N' is formed as (lm / N') * y: for a denormal N', y / N'
    // alone overflows.  lm == 0 (an underflowed weight) contributes nothing.
    float lN = lx[0];
    if (lm != 0.0f) {
      g[2] += lm * (k.y / c.phi - Np);
      float dN = -lm * c.phi;
      if (k.y != 0.0f) dN = dN + (lm / Np) * k.y;
      lN = lN + dN;
    }
    if (lN == 0.0f) {
      lx[0] = 0.0f;
      return;
    }
    // rproc: N' = r N e, e = exp(-N + sigma z); dN'/dN = r e (1 - N), formed
    // without dividing by N
    const float re = c.r * pp_expf(pp_fma(c.sigma, z[0], -N));
    g[0] += lN * (N * re) / c.r;
    g[1] += lN * Np * z[0];
    lx[0] = lN * re * (1.0f - N);
  }
  __device__ static void bwd_init(const Consts&, const float*, const float* lx0, float* g) {
    g[3] += lx0[0];
  }
};

// ---------------------------------------------------------------------------
// Model dispatch for LG: fn(Tag<M>{}) with M the instantiation for the
// model's dimensions -- compile-time dy for dx == dy <= 4, run-time dy <= 4
// otherwise up to 4 x 4, and the wide model (stride 9, run-time dy <= 9)
// when dx or dy is above 4.  Returns `none` when no instantiation applies
// (dimensions out of range, or a wide model where `wide` is false).
// ---------------------------------------------------------------------------
template <class M>
struct Tag {
  using type = M;
};

template <class R, class Fn>
R with_lg(const ppf_model& m, bool wide, R none, Fn&& fn) {
  if (m.dx <= 4 && m.dy <= 4) {
    switch (m.dx) {
      case 1: return m.dy == 1 ? fn(Tag<LG<1, 1>>{}) : fn(Tag<LG<1>>{});
      case 2: return m.dy == 2 ? fn(Tag<LG<2, 2>>{}) : fn(Tag<LG<2>>{});
      case 3: return m.dy == 3 ? fn(Tag<LG<3, 3>>{}) : fn(Tag<LG<3>>{});
      case 4: return m.dy == 4 ? fn(Tag<LG<4, 4>>{}) : fn(Tag<LG<4>>{});
      default: return none;
    }
  }
  if (!wide || m.dy < 1 || m.dy > 9) return none;
  switch (m.dx) {
    case 1: return fn(Tag<LG<1, 0, 9>>{});
    case 2: return fn(Tag<LG<2, 0, 9>>{});
    case 3: return fn(Tag<LG<3, 0, 9>>{});
    case 4: return fn(Tag<LG<4, 0, 9>>{});
    case 5: return fn(Tag<LG<5, 0, 9>>{});
    case 6: return fn(Tag<LG<6, 0, 9>>{});
    case 7: return fn(Tag<LG<7, 0, 9>>{});
    case 8: return fn(Tag<LG<8, 0, 9>>{});
    case 9: return fn(Tag<LG<9, 0, 9>>{});
    default: return none;
  }
}

}  // namespace ppf
