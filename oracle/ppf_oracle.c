/*
 * ppf_oracle.c -- C restatement of the particle-filter hot path with the CUDA
 * library's exact arithmetic.  TEST INFRASTRUCTURE ONLY: used by tests/, by
 * __graft_entry__.smoke() as the checker, and as bench.py's timed CPU baseline.
 *
 * It follows the reference's algorithm step by step --
 *   _pfilter_internal / _pfilter_step   pypomp/core/algorithms/pfilter.py:15-182
 *   _normalize_weights                  pypomp/core/algorithms/helpers.py:34-57
 *   _resample (systematic, side=right)  pypomp/core/algorithms/helpers.py:14-31
 *   _resampler (gather, -log J)         pypomp/core/algorithms/helpers.py:60-91
 *   _mop_internal / _mop_step           pypomp/core/algorithms/mop.py:19-135
 *   _perfilter_internal / scan body     pypomp/core/algorithms/mif.py:88-258
 *   _resampler_thetas                   pypomp/core/algorithms/helpers.py:103-141
 *   LG _rinit/_rproc/_dmeas             pypomp/models/linear_gaussian.py:139-177
 *   LG _rmeas                           pypomp/models/linear_gaussian.py:180-191
 *   _simulate_internal / _helper        pypomp/core/algorithms/simulate.py:15-142
 * -- but with the arithmetic definitions of include/ppf.h: float32 model math
 * in a fixed order, ppf_detmath.h elementary functions, the fixed-point CDF
 * summed sequentially in uint64, and ancestors found by a sequential
 * two-pointer merge of the systematic points with the CDF (the CUDA paths use
 * a closed-form offset per parent and a max-scan, or a binary search).  So the
 * CUDA results must match this file bit for bit: log-weights, ancestors,
 * particles; the float64 log-likelihood to rounding of log().
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off, no fast-math).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "ppf.h"
#include "ppf_detmath.h"
#include "ppf_philox.h"
#include "ppf_sample.h"

#define LOG2PI_F 1.83787706640934548356f

typedef unsigned __int128 u128;

/* LG dimensions up to 9 (pypomp/models/linear_gaussian.py:48 MAX_DIM): matrix
 * row stride, and the largest parameter count (LG 9 x 9: 81 + 81 + 45 + 45 + 9). */
#define LGS 9
#define MAXP 261

/* ------------------------------------------------------------------------ */
/* Models (same formulas and operation order as the CUDA device code)       */
/* ------------------------------------------------------------------------ */

typedef struct {
  int kind, dx, dy;
  float A[LGS * LGS], C[LGS * LGS], LQ[LGS * LGS], L[LGS * LGS], Linv[LGS], X0[LGS], c0,
        LR[LGS * LGS];  /* LG, row stride LGS */
  float kappa, theta, xi, rho, mu, v0, dt, sqdt, mudt, rhoc, svc0, kdt, xsq; /* SV */
  float r, sigma, phi, N0;                                         /* Ricker */
} consts_t;

static float tanh_det(float a) {
  const float e = pp_expf(-2.0f * fabsf(a));
  const float t = (1.0f - e) / (1.0f + e);
  return a < 0.0f ? -t : t;
}

static void prepare(consts_t* c, const float* th, const ppf_model* m, int est) {
  memset(c, 0, sizeof(*c));
  c->kind = m->kind; c->dx = m->dx; c->dy = m->dy;
  if (m->kind == PPF_MODEL_LG) {
    const int dx = m->dx, dy = m->dy;
    int p = 0;
    float* LR = c->LR;
    for (int i = 0; i < dx; ++i)
      for (int k = 0; k < dx; ++k) c->A[i * LGS + k] = th[p++];
    for (int i = 0; i < dy; ++i)
      for (int k = 0; k < dx; ++k) c->C[i * LGS + k] = th[p++];
    for (int i = 0; i < dx; ++i)
      for (int k = 0; k <= i; ++k) {
        float v = th[p++];
        if (est && i == k) v = pp_expf(v);
        c->LQ[i * LGS + k] = v;
      }
    for (int i = 0; i < dy; ++i)
      for (int k = 0; k <= i; ++k) {
        float v = th[p++];
        if (est && i == k) v = pp_expf(v);
        LR[i * LGS + k] = v;
      }
    for (int i = 0; i < dx; ++i) c->X0[i] = th[p++];
    float R[LGS * LGS] = {0};
    for (int i = 0; i < dy; ++i)
      for (int k = 0; k <= i; ++k) {
        float s = 0.0f;
        for (int l = 0; l <= k; ++l) s = s + LR[i * LGS + l] * LR[k * LGS + l];
        R[i * LGS + k] = s;
      }
    for (int i = 0; i < dy; ++i)
      for (int k = 0; k <= i; ++k) {
        float s = R[i * LGS + k];
        for (int l = 0; l < k; ++l) s = s - c->L[i * LGS + l] * c->L[k * LGS + l];
        if (i == k) c->L[i * LGS + i] = sqrtf(s);
        else c->L[i * LGS + k] = s / c->L[k * LGS + k];
      }
    float c0 = -0.5f * (float)dy * LOG2PI_F;
    for (int i = 0; i < dy; ++i) {
      c->Linv[i] = 1.0f / c->L[i * LGS + i];
      c0 = c0 - pp_logf(c->L[i * LGS + i]);
    }
    c->c0 = c0;
  } else if (m->kind == PPF_MODEL_SV) {
    c->kappa = est ? pp_expf(th[0]) : th[0];
    c->theta = est ? pp_expf(th[1]) : th[1];
    c->xi = est ? pp_expf(th[2]) : th[2];
    c->rho = est ? tanh_det(th[3]) : th[3];
    c->mu = th[4];
    c->v0 = th[5];
    c->dt = m->dt;
    c->sqdt = sqrtf(m->dt);
    c->mudt = c->mu * c->dt;
    c->rhoc = sqrtf(1.0f - c->rho * c->rho);
    c->svc0 = -0.5f * LOG2PI_F - pp_logf(c->rhoc) - 0.5f * pp_logf(c->dt);
    c->kdt = c->kappa * c->dt;
    c->xsq = c->xi * c->sqdt;
  } else {
    c->r = est ? pp_expf(th[0]) : th[0];
    c->sigma = est ? pp_expf(th[1]) : th[1];
    c->phi = est ? pp_expf(th[2]) : th[2];
    c->N0 = est ? pp_expf(th[3]) : th[3];
  }
}

static int n_init(const consts_t* c) { return c->kind == PPF_MODEL_LG ? c->dx : 0; }
static int n_step(const consts_t* c) { return c->kind == PPF_MODEL_LG ? c->dx : 1; }

static void rinit(const consts_t* c, const float* z, float* x) {
  if (c->kind == PPF_MODEL_LG) {
    for (int i = 0; i < c->dx; ++i) {
      float acc = c->X0[i];
      for (int k = 0; k <= i; ++k) acc = fmaf(c->LQ[i * LGS + k], z[k], acc);
      x[i] = acc;
    }
  } else if (c->kind == PPF_MODEL_SV) {
    x[0] = c->v0;
    x[1] = 0.0f;
  } else {
    x[0] = c->N0;
  }
}

static void rproc(const consts_t* c, float* x, const float* z) {
  if (c->kind == PPF_MODEL_LG) {
    float y[LGS];
    for (int i = 0; i < c->dx; ++i) {
      float acc = 0.0f;
      for (int k = 0; k < c->dx; ++k) acc = fmaf(c->A[i * LGS + k], x[k], acc);
      for (int k = 0; k <= i; ++k) acc = fmaf(c->LQ[i * LGS + k], z[k], acc);
      y[i] = acc;
    }
    for (int i = 0; i < c->dx; ++i) x[i] = y[i];
  } else if (c->kind == PPF_MODEL_SV) {
    const float v = x[0];
    const float emh = pp_expf(-0.5f * v);
    const float emv = emh * emh;
    const float a1 = fmaf(c->theta, emv, -1.0f);
    const float v1 = fmaf(c->kdt, a1, v);
    x[0] = fmaf(c->xsq * emh, z[0], v1);
    x[1] = z[0];
  } else {
    const float N = x[0];
    x[0] = (c->r * N) * pp_expf(fmaf(c->sigma, z[0], -N));
  }
}

static float dmeas(const consts_t* c, const float* y, float ycon, const float* x) {
  if (c->kind == PPF_MODEL_LG) {
    float s[LGS];
    float q = 0.0f;
    for (int i = 0; i < c->dy; ++i) {
      float a = 0.0f;
      for (int k = 0; k < c->dx; ++k) a = fmaf(c->C[i * LGS + k], x[k], a);
      float r = y[i] - a;
      for (int l = 0; l < i; ++l) r = fmaf(-c->L[i * LGS + l], s[l], r);
      s[i] = r * c->Linv[i];
      q = fmaf(s[i], s[i], q);
    }
    return fmaf(-0.5f, q, c->c0);
  } else if (c->kind == PPF_MODEL_SV) {
    const float v = x[0];
    const float sd = pp_expf(0.5f * v) * c->sqdt;
    const float mean = fmaf(c->rho * sd, x[1], c->mudt);
    const float r = (y[0] - mean) / (c->rhoc * sd);
    return fmaf(-0.5f * r, r, fmaf(-0.5f, v, c->svc0));
  } else {
    const float lam = c->phi * x[0];
    if (y[0] == 0.0f) return -lam;
    return fmaf(y[0], pp_logf(lam), -lam) - ycon;
  }
}

/* ------------------------------------------------------------------------ */
/* Filter loop                                                              */
/* ------------------------------------------------------------------------ */

static void noise(const ppf_pfilter_desc* d, int f, int j, int s, int n, float* z) {
  if (d->flags & PPF_F_INJECT) {
    if (s == 0) {
      for (int i = 0; i < n; ++i) z[i] = d->inj_z0[((size_t)f * d->J + j) * n + i];
    } else {
      const size_t base = (((size_t)f * d->T + (s - 1)) * d->J + j) * n;
      for (int i = 0; i < n; ++i) z[i] = d->inj_z[base + i];
    }
  } else {
    pp_normals(d->seeds[f], (uint32_t)j, (uint32_t)s, PPF_TAG_PROCESS, n, z);
  }
}

static uint32_t uniform32(const ppf_pfilter_desc* d, int f, int t) {
  if (d->flags & PPF_F_INJECT) return pp_u32_from_float(d->inj_u[(size_t)f * d->T + t]);
  return pp_resample_u32(d->seeds[f], (uint32_t)(t + 1));
}

static float propagate(const ppf_pfilter_desc* d, const consts_t* c, int f, int u, int j, int t, float* x) {
  float z[LGS];
  noise(d, f, j, t + 1, n_step(c), z);
  rproc(c, x, z);
  const float* y = d->ys + ((size_t)u * d->T + t) * d->model.dy;
  const float yc = d->ycon ? d->ycon[(size_t)u * d->T + t] : 0.0f;
  return dmeas(c, y, yc, x);
}

/* One filter.  mop != 0: resampling weights are the measurement densities
 * alone (mop.py:120) and the log-likelihood term subtracts log J. */
static void run_filter(const ppf_pfilter_desc* d, int f, int mop) {
  const int J = d->J, dx = d->model.dx;
  const int u = d->unit ? d->unit[f] : 0;
  const int Tf = d->T_u ? d->T_u[u] : d->T;
  consts_t c;
  prepare(&c, d->theta + (size_t)f * d->model.n_params, &d->model, (d->flags & PPF_F_EST) != 0);
  const float base_init = pp_logf(1.0f / (float)J);
  const float base_rs = -pp_logf((float)J);
  const float logthresh = d->thresh > 0.0f ? pp_logf(d->thresh) : -INFINITY;
  float* x = (float*)malloc(sizeof(float) * dx * J);
  float* xn = (float*)malloc(sizeof(float) * dx * J);
  float* w = (float*)malloc(sizeof(float) * J);
  float* wn = (float*)malloc(sizeof(float) * J);
  uint64_t* C = (uint64_t*)malloc(sizeof(uint64_t) * J);
  int* par = (int*)malloc(sizeof(int) * J);
  for (int j = 0; j < J; ++j) {
    float z[LGS], xj[LGS];
    noise(d, f, j, 0, n_init(&c), z);
    rinit(&c, z, xj);
    const float m = propagate(d, &c, f, u, j, 0, xj);
    for (int k = 0; k < dx; ++k) x[k * J + j] = xj[k];
    w[j] = (mop ? 0.0f : base_init) + m;
  }
  double loglik = 0.0;
  for (int t = 0; t < Tf; ++t) {
    if (d->logw) memcpy(d->logw + ((size_t)f * d->T + t) * J, w, sizeof(float) * J);
    /* max / min over finite weights; NaN or +inf marks the filter */
    int nanf = 0;
    float Mx = -INFINITY, mn = INFINITY;
    for (int j = 0; j < J; ++j) {
      if (w[j] != w[j] || w[j] == INFINITY) { nanf = 1; continue; }
      if (w[j] > Mx) Mx = w[j];
      if (w[j] < mn) mn = w[j];
    }
    const int collapsed = !nanf && Mx == -INFINITY;
    const int qc = nanf || Mx == -INFINITY;
    uint64_t tot = 0;
    double s2 = 0.0, fx[LGS] = {0}, px[LGS] = {0};
    for (int j = 0; j < J; ++j) {
      uint64_t q;
      double e;
      if (qc) { q = 1; e = 1.0; }
      else if (w[j] != w[j]) { q = 0; e = 0.0; }
      else {
        const float ef = pp_expf(w[j] - Mx);
        q = (uint64_t)llrintf(ef * 1099511627776.0f);
        e = (double)ef;
      }
      tot += q;
      C[j] = tot;
      s2 += e * e;
      for (int k = 0; k < dx; ++k) {
        fx[k] += (double)x[k * J + j] * e;
        px[k] += (double)x[k * J + j];
      }
    }
    double ll;
    if (nanf) ll = NAN;
    else if (collapsed) ll = -INFINITY;
    else ll = (double)Mx + log((double)tot) - 40.0 * 0.69314718055994530942 - (mop ? log((double)J) : 0.0);
    loglik += ll;
    if ((d->flags & PPF_F_CLL) && d->cll) d->cll[(size_t)f * d->T + t] = ll;
    const double S1 = (double)tot * 9.094947017729282e-13;
    if ((d->flags & PPF_F_ESS) && d->ess)
      d->ess[(size_t)f * d->T + t] = nanf ? NAN : (collapsed ? (float)J : (float)(S1 * S1 / s2));
    for (int k = 0; k < dx; ++k) {
      if ((d->flags & PPF_F_FMEAN) && d->fmean)
        d->fmean[((size_t)f * d->T + t) * dx + k] = (float)(collapsed ? px[k] / J : fx[k] / S1);
      if ((d->flags & PPF_F_PMEAN) && d->pmean)
        d->pmean[((size_t)f * d->T + t) * dx + k] = (float)(px[k] / J);
    }
    const int last = (t == Tf - 1);
    if (last && !d->anc) break;
    int rs;
    if (nanf) rs = 0;
    else if (Mx == -INFINITY) rs = 0.0f > logthresh;
    else rs = (Mx - mn) > logthresh;
    if (rs) {
      /* systematic resampling: child k takes the first parent whose CDF
       * exceeds its point, i.e. #{ j : C_j J 2^32 <= (u32 + k 2^32) tot } */
      const uint32_t u32 = uniform32(d, f, t);
      const u128 Jsh = (u128)((uint64_t)J << 32);
      int j = 0;
      for (int k = 0; k < J; ++k) {
        const u128 R = ((u128)u32 + ((u128)k << 32)) * (u128)tot;
        while (j < J && (u128)C[j] * Jsh <= R) ++j;
        par[k] = j;
      }
    } else {
      for (int k = 0; k < J; ++k) par[k] = k;
    }
    if (d->anc) memcpy(d->anc + ((size_t)f * d->T + t) * J, par, sizeof(int) * J);
    if (last) break;
    float lt32 = 0.0f;
    if (!rs) {
      if (nanf) lt32 = NAN;
      else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
    }
    for (int k = 0; k < J; ++k) {
      float xk[LGS];
      for (int q = 0; q < dx; ++q) xk[q] = x[q * J + par[k]];
      float b;
      if (rs) b = mop ? 0.0f : base_rs;
      else b = collapsed ? -pp_logf((float)J) : w[k] - lt32;
      const float m = propagate(d, &c, f, u, k, t + 1, xk);
      for (int q = 0; q < dx; ++q) xn[q * J + k] = xk[q];
      wn[k] = b + m;
    }
    float* tmp = x; x = xn; xn = tmp;
    float* tw = w; w = wn; wn = tw;
  }
  d->loglik[f] = loglik;
  free(x); free(xn); free(w); free(wn); free(C); free(par);
}

typedef struct {
  const ppf_pfilter_desc* d;
  int mop, tid, nthreads;
} job_t;

static void* worker(void* arg) {
  const job_t* jb = (const job_t*)arg;
  for (int f = jb->tid; f < jb->d->F; f += jb->nthreads) run_filter(jb->d, f, jb->mop);
  return NULL;
}

/* Runs the F filters of `d` (all pointers HOST memory); `nthreads` > 1
 * spreads whole filters over POSIX threads. */
int ppfo_pfilter(const ppf_pfilter_desc* d, int mop, int nthreads) {
  if (!d || d->J < 1 || d->F < 1 || d->T < 1) return PPF_EINVAL;
  if (nthreads <= 1 || d->F == 1) {
    for (int f = 0; f < d->F; ++f) run_filter(d, f, mop);
    return PPF_OK;
  }
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  job_t jobs[256];
  for (int i = 0; i < nthreads; ++i) {
    jobs[i].d = d; jobs[i].mop = mop; jobs[i].tid = i; jobs[i].nthreads = nthreads;
    pthread_create(&th[i], NULL, worker, &jobs[i]);
  }
  for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
  return PPF_OK;
}

/* MOP-alpha surrogate for gradient checks (mop.py:69-135 as a function of
 * theta with the discrete choices frozen): ancestors anc[F][T][J] are given,
 * and stop_gradient(m) is the constant m0[F][T][J] recorded at the base
 * parameters (pass m0_in = NULL to record it into m0_out).  In float64:
 *   wP = alpha wF;  ll_t = LSE(wP + m) - LSE(wP);  wF = (wP + m - m0)[anc]
 * value[f] = -sum_t ll_t.  At the base parameters it equals the MOP value; its
 * derivative there is the MOP-alpha gradient. */
static double lse(const double* v, int n) {
  double mx = -INFINITY;
  for (int i = 0; i < n; ++i) mx = v[i] > mx ? v[i] : mx;
  if (!(mx > -INFINITY)) return mx;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += exp(v[i] - mx);
  return mx + log(s);
}

/* DPOP adds, per step, the predicted state's component pwi as
 * pw - stop_gradient(pw) to the carried weights (dpop.py:203-209):
 *   wP = alpha wF + pw - p0
 * with p0[F][T][J] the frozen pw (p0_in, or recorded into p0_out).  pwi < 0
 * is MOP-alpha. */
static int surrogate_impl(const ppf_pfilter_desc* d, float alpha, int pwi, const int* anc,
                          const float* m0_in, float* m0_out, const float* p0_in, float* p0_out,
                          double* value) {
  const int J = d->J, dx = d->model.dx, T = d->T;
  for (int f = 0; f < d->F; ++f) {
    const int u = d->unit ? d->unit[f] : 0;
    consts_t c;
    prepare(&c, d->theta + (size_t)f * d->model.n_params, &d->model, (d->flags & PPF_F_EST) != 0);
    float* x = (float*)malloc(sizeof(float) * dx * J);
    float* xp = (float*)malloc(sizeof(float) * dx * J);
    double* wF = (double*)malloc(sizeof(double) * J);
    double* wP = (double*)malloc(sizeof(double) * J);
    double* v = (double*)malloc(sizeof(double) * J);
    float* m = (float*)malloc(sizeof(float) * J);
    for (int j = 0; j < J; ++j) {
      float z[LGS], xj[LGS];
      noise(d, f, j, 0, n_init(&c), z);
      rinit(&c, z, xj);
      for (int k = 0; k < dx; ++k) x[k * J + j] = xj[k];
      wF[j] = -log((double)J);
    }
    double ll = 0.0;
    for (int t = 0; t < T; ++t) {
      const size_t row = ((size_t)f * T + t) * J;
      for (int j = 0; j < J; ++j) {
        wP[j] = (double)alpha * wF[j];
        float xj[LGS];
        for (int k = 0; k < dx; ++k) xj[k] = x[k * J + j];
        m[j] = propagate(d, &c, f, u, j, t, xj);
        for (int k = 0; k < dx; ++k) xp[k * J + j] = xj[k];
        if (pwi >= 0) {
          const float pw = xj[pwi];
          if (!p0_in && p0_out) p0_out[row + j] = pw;
          wP[j] += (double)pw - (double)(p0_in ? p0_in[row + j] : pw);
        }
        v[j] = wP[j] + (double)m[j];
      }
      const double a1 = lse(v, J), a2 = lse(wP, J);
      ll += a1 - a2;
      const float* m0 = m0_in ? m0_in + ((size_t)f * T + t) * J : m;
      if (!m0_in && m0_out) memcpy(m0_out + ((size_t)f * T + t) * J, m, sizeof(float) * J);
      const int* at = anc + ((size_t)f * T + t) * J;
      for (int k = 0; k < J; ++k) {
        const int j = at[k];
        for (int q = 0; q < dx; ++q) x[q * J + k] = xp[q * J + j];
        v[k] = wP[j] + (double)m[j] - (double)m0[j];
      }
      memcpy(wF, v, sizeof(double) * J);
    }
    value[f] = -ll;
    free(x); free(xp); free(wF); free(wP); free(v); free(m);
  }
  return PPF_OK;
}

int ppfo_mop_surrogate(const ppf_pfilter_desc* d, float alpha, const int* anc, const float* m0_in,
                       float* m0_out, double* value) {
  return surrogate_impl(d, alpha, -1, anc, m0_in, m0_out, NULL, NULL, value);
}

int ppfo_dpop_surrogate(const ppf_pfilter_desc* d, float alpha, int pwi, const int* anc,
                        const float* m0_in, float* m0_out, const float* p0_in, float* p0_out,
                        double* value) {
  if (pwi < 0 || pwi >= d->model.dx) return PPF_EINVAL;
  return surrogate_impl(d, alpha, pwi, anc, m0_in, m0_out, p0_in, p0_out, value);
}

/* ------------------------------------------------------------------------ */
/* IF2 perturbed filter (mif.py:88-258)                                     */
/* ------------------------------------------------------------------------ */

static void if2_noise(const ppf_perfilter_desc* d, int f, int j, int s, int n, float* z) {
  if (n <= 0) return;
  if (d->flags & PPF_F_INJECT) {
    if (s == 0) {
      for (int i = 0; i < n; ++i) z[i] = d->inj_z0[((size_t)f * d->J + j) * n + i];
    } else {
      const size_t base = (((size_t)f * d->T + (s - 1)) * d->J + j) * n;
      for (int i = 0; i < n; ++i) z[i] = d->inj_z[base + i];
    }
  } else {
    pp_normals(d->seeds[f], (uint32_t)j, (uint32_t)s, PPF_TAG_PROCESS, n, z);
  }
}

/* P perturbation normals of particle j: s = 0 before rinit, s = t + 1 before step t. */
static void if2_perturb_noise(const ppf_perfilter_desc* d, int f, int j, int s, int P, float* z) {
  if (d->flags & PPF_F_INJECT) {
    const float* src = (s == 0) ? d->inj_zp0 + ((size_t)f * d->J + j) * P
                                : d->inj_zp + (((size_t)f * d->T + (s - 1)) * d->J + j) * P;
    for (int i = 0; i < P; ++i) z[i] = src[i];
  } else {
    pp_normals(d->seeds[f], (uint32_t)j, (uint32_t)s, PPF_TAG_PERTURB, P, z);
  }
}

/* jnp.nan_to_num(m, nan=log(1e-18)) (mif.py:205-210) */
static float if2_measure(float m) {
  if (m != m) return pp_logf(1e-18f);
  if (m == INFINITY) return 3.4028234663852886e38f;
  if (m == -INFINITY) return -3.4028234663852886e38f;
  return m;
}

/* Perturb th (P values) with sds sig * cool, then step the particle:
 * rproc with process normals of counter s, dmeas at observation t. */
static float if2_step(const ppf_perfilter_desc* d, int f, int u, int j, int t, int s, float cool,
                      float* th, float* x) {
  const int P = d->model.n_params;
  float zp[MAXP];
  if2_perturb_noise(d, f, j, s, P, zp);
  for (int p = 0; p < P; ++p) th[p] = th[p] + (cool * d->rw_sig[p]) * zp[p];
  consts_t c;
  prepare(&c, th, &d->model, !(d->flags & PPF_F_NATURAL));
  float z[LGS];
  if2_noise(d, f, j, s, n_step(&c), z);
  rproc(&c, x, z);
  const float* y = d->ys + ((size_t)u * d->T + t) * d->model.dy;
  const float yc = d->ycon ? d->ycon[(size_t)u * d->T + t] : 0.0f;
  return if2_measure(dmeas(&c, y, yc, x));
}

static void run_perfilter(const ppf_perfilter_desc* d, int f) {
  const int J = d->J, dx = d->model.dx, P = d->model.n_params;
  const int u = d->unit ? d->unit[f] : 0;
  const int Tf = d->T_u ? d->T_u[u] : d->T;
  const float base_init = pp_logf(1.0f / (float)J);
  const float base_rs = -pp_logf((float)J);
  const float logthresh = d->thresh > 0.0f ? pp_logf(d->thresh) : -INFINITY;
  const float* cool = d->cool + (size_t)u * d->T;
  float* x = (float*)malloc(sizeof(float) * dx * J);
  float* xn = (float*)malloc(sizeof(float) * dx * J);
  float* th = (float*)malloc(sizeof(float) * P * J);
  float* thn = (float*)malloc(sizeof(float) * P * J);
  float* w = (float*)malloc(sizeof(float) * J);
  float* wn = (float*)malloc(sizeof(float) * J);
  uint64_t* C = (uint64_t*)malloc(sizeof(uint64_t) * J);
  int* par = (int*)malloc(sizeof(int) * J);
  const float* S = d->swarm_in + (size_t)f * P * J;
  for (int j = 0; j < J; ++j) {
    float tj[MAXP], zp[MAXP], z[LGS], xj[LGS];
    for (int p = 0; p < P; ++p) tj[p] = S[(size_t)p * J + j];
    if2_perturb_noise(d, f, j, 0, P, zp);
    for (int p = 0; p < P; ++p) tj[p] = tj[p] + (d->cool0[u] * d->rw_sig0[p]) * zp[p];
    consts_t c;
    prepare(&c, tj, &d->model, !(d->flags & PPF_F_NATURAL));
    if2_noise(d, f, j, 0, n_init(&c), z);
    rinit(&c, z, xj);
    const float m = if2_step(d, f, u, j, 0, 1, cool[0], tj, xj);
    for (int k = 0; k < dx; ++k) x[k * J + j] = xj[k];
    for (int p = 0; p < P; ++p) th[(size_t)p * J + j] = tj[p];
    w[j] = base_init + m;
  }
  double loglik = 0.0;
  for (int t = 0; t < Tf; ++t) {
    int nanf = 0;
    float Mx = -INFINITY, mn = INFINITY;
    for (int j = 0; j < J; ++j) {
      if (w[j] != w[j] || w[j] == INFINITY) { nanf = 1; continue; }
      if (w[j] > Mx) Mx = w[j];
      if (w[j] < mn) mn = w[j];
    }
    const int collapsed = !nanf && Mx == -INFINITY;
    const int qc = nanf || Mx == -INFINITY;
    uint64_t tot = 0;
    for (int j = 0; j < J; ++j) {
      uint64_t q;
      if (qc) q = 1;
      else if (w[j] != w[j]) q = 0;
      else q = (uint64_t)llrintf(pp_expf(w[j] - Mx) * 1099511627776.0f);
      tot += q;
      C[j] = tot;
    }
    double ll;
    if (nanf) ll = NAN;
    else if (collapsed) ll = -INFINITY;
    else ll = (double)Mx + log((double)tot) - 40.0 * 0.69314718055994530942;
    loglik += ll;
    if ((d->flags & PPF_F_CLL) && d->cll) d->cll[(size_t)f * d->T + t] = ll;
    int rs;
    if (nanf) rs = 0;
    else if (Mx == -INFINITY) rs = 0.0f > logthresh;
    else rs = (Mx - mn) > logthresh;
    if (rs) {
      const uint32_t u32 = (d->flags & PPF_F_INJECT) ? pp_u32_from_float(d->inj_u[(size_t)f * d->T + t])
                                                     : pp_resample_u32(d->seeds[f], (uint32_t)(t + 1));
      const u128 Jsh = (u128)((uint64_t)J << 32);
      int j = 0;
      for (int k = 0; k < J; ++k) {
        const u128 R = ((u128)u32 + ((u128)k << 32)) * (u128)tot;
        while (j < J && (u128)C[j] * Jsh <= R) ++j;
        par[k] = j;
      }
    } else {
      for (int k = 0; k < J; ++k) par[k] = k;
    }
    if ((d->flags & PPF_F_SAVE_ANC) && d->anc) memcpy(d->anc + ((size_t)f * d->T + t) * J, par, sizeof(int) * J);
    if (t == Tf - 1) {
      float* out = d->swarm_out + (size_t)f * P * J;
      for (int k = 0; k < J; ++k)
        for (int p = 0; p < P; ++p) out[(size_t)p * J + k] = th[(size_t)p * J + par[k]];
      break;
    }
    float lt32 = 0.0f;
    if (!rs) {
      if (nanf) lt32 = NAN;
      else if (!collapsed) lt32 = Mx + pp_logf((float)tot * 9.094947017729282e-13f);
    }
    for (int k = 0; k < J; ++k) {
      float xk[LGS], tk[MAXP];
      for (int q = 0; q < dx; ++q) xk[q] = x[q * J + par[k]];
      for (int p = 0; p < P; ++p) tk[p] = th[(size_t)p * J + par[k]];
      float b;
      if (rs) b = base_rs;
      else b = collapsed ? -pp_logf((float)J) : w[k] - lt32;
      const float m = if2_step(d, f, u, k, t + 1, t + 2, cool[t + 1], tk, xk);
      for (int q = 0; q < dx; ++q) xn[q * J + k] = xk[q];
      for (int p = 0; p < P; ++p) thn[(size_t)p * J + k] = tk[p];
      wn[k] = b + m;
    }
    float* tmp = x; x = xn; xn = tmp;
    float* tt = th; th = thn; thn = tt;
    float* tw = w; w = wn; wn = tw;
  }
  d->loglik[f] = loglik;
  free(x); free(xn); free(th); free(thn); free(w); free(wn); free(C); free(par);
}

typedef struct {
  const ppf_perfilter_desc* d;
  int tid, nthreads;
} if2_job_t;

static void* if2_worker(void* arg) {
  const if2_job_t* jb = (const if2_job_t*)arg;
  for (int f = jb->tid; f < jb->d->F; f += jb->nthreads) run_perfilter(jb->d, f);
  return NULL;
}

/* Runs the F perturbed filters of `d` (all pointers HOST memory). */
int ppfo_perfilter(const ppf_perfilter_desc* d, int nthreads) {
  if (!d || d->J < 1 || d->F < 1 || d->T < 1 || d->model.n_params > MAXP) return PPF_EINVAL;
  if (nthreads <= 1 || d->F == 1) {
    for (int f = 0; f < d->F; ++f) run_perfilter(d, f);
    return PPF_OK;
  }
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  if2_job_t jobs[256];
  for (int i = 0; i < nthreads; ++i) {
    jobs[i].d = d; jobs[i].tid = i; jobs[i].nthreads = nthreads;
    pthread_create(&th[i], NULL, if2_worker, &jobs[i]);
  }
  for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
  return PPF_OK;
}

/* ------------------------------------------------------------------------ */
/* Simulation                                                               */
/* ------------------------------------------------------------------------ */

/* Observation draw of replicate k at step s (linear_gaussian.py:180-191 for
 * LG: y = C x + L_R w; SV: the conditional normal of the return given eps;
 * Ricker: Poisson(phi N)). */
static void rmeas(const consts_t* c, const float* x, uint64_t seed, uint32_t k, uint32_t s, float* y) {
  if (c->kind == PPF_MODEL_LG) {
    float w[LGS];
    pp_normals(seed, k, s, PPF_TAG_MEASURE, c->dy, w);
    for (int i = 0; i < c->dy; ++i) {
      float a = 0.0f;
      for (int q = 0; q < c->dx; ++q) a = fmaf(c->C[i * LGS + q], x[q], a);
      for (int l = 0; l <= i; ++l) a = fmaf(c->LR[i * LGS + l], w[l], a);
      y[i] = a;
    }
  } else if (c->kind == PPF_MODEL_SV) {
    float w[1];
    pp_normals(seed, k, s, PPF_TAG_MEASURE, 1, w);
    const float sd = pp_expf(0.5f * x[0]) * c->sqdt;
    const float mean = fmaf(c->rho * sd, x[1], c->mudt);
    y[0] = fmaf(c->rhoc * sd, w[0], mean);
  } else {
    y[0] = pp_poisson(c->phi * x[0], seed, k, s);
  }
}

/* Trajectories of F parameter sets x nsim replicates (all pointers HOST
 * memory, layouts of ppf_simulate_desc): rinit from the process normals of
 * step 0, then per observation t the process normals of step t + 1 (rproc)
 * and the measurement draws of step t + 1 (rmeas). */
int ppfo_simulate(const ppf_simulate_desc* d) {
  if (!d || d->F < 1 || d->nsim < 1 || d->T < 0 || !d->X || (d->T > 0 && !d->Y)) return PPF_EINVAL;
  const int dx = d->model.dx, dy = d->model.dy, P = d->model.n_params;
  for (int f = 0; f < d->F; ++f) {
    consts_t c;
    prepare(&c, d->theta + (size_t)f * P, &d->model, (d->flags & PPF_F_EST) != 0);
    const uint64_t seed = d->seeds[f];
    for (int k = 0; k < d->nsim; ++k) {
      float* X = d->X + ((size_t)f * d->nsim + k) * (size_t)(d->T + 1) * dx;
      float* Y = d->Y ? d->Y + ((size_t)f * d->nsim + k) * (size_t)d->T * dy : NULL;
      float x[LGS], z[LGS];
      const int n0 = n_init(&c), n1 = n_step(&c);
      if (n0 > 0) pp_normals(seed, (uint32_t)k, 0u, PPF_TAG_PROCESS, n0, z);
      rinit(&c, z, x);
      for (int i = 0; i < dx; ++i) X[i] = x[i];
      for (int t = 0; t < d->T; ++t) {
        pp_normals(seed, (uint32_t)k, (uint32_t)(t + 1), PPF_TAG_PROCESS, n1, z);
        rproc(&c, x, z);
        rmeas(&c, x, seed, (uint32_t)k, (uint32_t)(t + 1), Y + (size_t)t * dy);
        for (int i = 0; i < dx; ++i) X[(size_t)(t + 1) * dx + i] = x[i];
      }
    }
  }
  return PPF_OK;
}

float ppfo_poisson(float lam, uint64_t seed, uint32_t k, uint32_t s) { return pp_poisson(lam, seed, k, s); }
float ppfo_logfact(float k) { return pp_logfact(k); }

/* Elementary functions and Philox, exported for the tests that pin them. */
float ppfo_expf(float x) { return pp_expf(x); }
float ppfo_expq(float x) { return pp_expq(x); }
float ppfo_logf(float x) { return pp_logf(x); }
void ppfo_sincos2pif(float u, float* s, float* c) { pp_sincos2pif(u, s, c); }
void ppfo_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  const pp_u32x4 r = pp_philox4x32_10(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}
void ppfo_normals(uint64_t seed, uint32_t j, uint32_t s, uint32_t tag, int n, float* z) {
  pp_normals(seed, j, s, tag, n, z);
}
