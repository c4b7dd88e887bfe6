/*
 * ppf_detmath.h -- deterministic float32 elementary functions.
 *
 * The particle-filter kernels and the C oracle must produce bit-identical
 * float32 log-weights, so that resampling indices can be compared exactly.
 * Every function here is built only from IEEE-754 operations that are
 * correctly rounded on both the host (C99, no contraction) and the device
 * (sm_100a, compiled with -fmad=false): +, -, *, /, sqrtf, fmaf, rintf,
 * floorf and exponent-field bit manipulation.  No libm or CUDA math-library
 * routine is called, so host and device agree exactly.
 *
 * Methods (all from the mathematics, no library constants):
 *   pp_expf   Cody & Waite (1980) argument reduction x = k ln2 + r with a
 *             two-part ln2, then the Taylor series of e^r to degree 7
 *             (|r| <= ln2/2, truncation < 6e-9 relative), scaled by 2^k.
 *   pp_logf   x = m 2^e with m in [sqrt(1/2), sqrt(2)); log(m) = log(1+f),
 *             f = m - 1, by the division-free polynomial pp_log1p_red
 *             (least-squares fit on Chebyshev nodes, see there), plus e ln2
 *             with the two-part ln2.
 *   pp_sincos2pif  sin/cos of 2 pi u for u in [0,1): exact octant reduction
 *             of u, then Taylor series of sin and cos on [0, pi/4].
 * Accuracy (checked against double-precision libm in tests): <= 2 ulp.
 */
#ifndef PPF_DETMATH_H
#define PPF_DETMATH_H

#include <stdint.h>
#include <math.h>
#include <string.h>

#if defined(__CUDACC__)
#define PPF_HD __host__ __device__ __forceinline__
#else
#define PPF_HD static inline
#endif

PPF_HD uint32_t pp_f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}

PPF_HD float pp_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f; memcpy(&f, &u, 4); return f;
#endif
}

PPF_HD float pp_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}

PPF_HD float pp_rint(float x) {
#if defined(__CUDA_ARCH__)
  return rintf(x);
#else
  return rintf(x);
#endif
}

/* 2^n as a float for n in [-126, 127]. */
PPF_HD float pp_pow2i(int n) { return pp_u2f((uint32_t)(n + 127) << 23); }

PPF_HD float pp_expf(float x) {
  /* special cases are selected at the end so the main path has no branches */
  const float xc = fminf(fmaxf(x, -103.97208404541016f), 88.72283935546875f);
  const float k = pp_rint(xc * 1.44269502162933349609375f);       /* x / ln2 */
  float r = pp_fma(-k, 0.693145751953125f, xc);                     /* ln2 hi (16 bits) */
  r = pp_fma(-k, 1.428606765330187045e-06f, r);                      /* ln2 - hi */
  float p = 1.98412698412698413e-04f;                                /* 1/7! */
  p = pp_fma(p, r, 1.38888888888888889e-03f);                        /* 1/6! */
  p = pp_fma(p, r, 8.33333333333333333e-03f);                        /* 1/5! */
  p = pp_fma(p, r, 4.16666666666666667e-02f);                        /* 1/4! */
  p = pp_fma(p, r, 1.66666666666666667e-01f);                        /* 1/3! */
  p = pp_fma(p, r, 0.5f);
  p = pp_fma(p, r, 1.0f);
  p = pp_fma(p, r, 1.0f);
  const int ki = (int)k;
  const int k1 = ki >> 1;                                            /* floor(k/2) */
  const int k2 = ki - k1;
  float y = (p * pp_pow2i(k1)) * pp_pow2i(k2);
  y = (x > 88.72283935546875f) ? pp_u2f(0x7f800000u) : y;
  y = (x < -103.97208404541016f) ? 0.0f : y;
  return (x != x) ? x : y;
}

/* pp_expf restricted to the weight quantiser's range: for x in [-32, 0] it
 * returns exactly pp_expf(x) (there k = rint(x / ln2) lies in [-47, 0], so the
 * two half-scalings of pp_expf are one exact scaling by 2^k), and 0 below
 * -32, where pp_expf(x) < 2^-46 and rint(e 2^40) is 0 either way.  NaN and
 * +inf inputs are the caller's to handle. */
PPF_HD float pp_expq(float x) {
  const float k = pp_rint(x * 1.44269502162933349609375f);
  float r = pp_fma(-k, 0.693145751953125f, x);
  r = pp_fma(-k, 1.428606765330187045e-06f, r);
  float p = 1.98412698412698413e-04f;
  p = pp_fma(p, r, 1.38888888888888889e-03f);
  p = pp_fma(p, r, 8.33333333333333333e-03f);
  p = pp_fma(p, r, 4.16666666666666667e-02f);
  p = pp_fma(p, r, 1.66666666666666667e-01f);
  p = pp_fma(p, r, 0.5f);
  p = pp_fma(p, r, 1.0f);
  p = pp_fma(p, r, 1.0f);
  const int ki = (int)k;
  const float y = p * pp_pow2i(ki < -126 ? -126 : ki);
  return (x < -32.0f) ? 0.0f : y;
}

/* log(1+f) for f in [sqrt(1/2)-1, sqrt(2)-1] as f - f^2/2 + f^3 R(f), R a
 * degree-8 polynomial fitted by least squares on Chebyshev nodes of the
 * interval (float64 fit, coefficients rounded to float32); < 0.75 ulp. */
PPF_HD float pp_log1p_red(float f) {
  float p = 0.07148932665586472f;
  p = pp_fma(p, f, -0.1157151460647583f);
  p = pp_fma(p, f, 0.1166200265288353f);
  p = pp_fma(p, f, -0.12411021441221237f);
  p = pp_fma(p, f, 0.14249871671199799f);
  p = pp_fma(p, f, -0.1666848063468933f);
  p = pp_fma(p, f, 0.2000070959329605f);
  p = pp_fma(p, f, -0.24999989569187164f);
  p = pp_fma(p, f, 0.3333333134651184f);
  const float f2 = f * f;
  const float f3 = f2 * f;
  return f + pp_fma(f3, p, -0.5f * f2);
}

PPF_HD float pp_logf(float x) {
  /* main path on a safe input; special cases selected at the end */
  const int sub = x < 1.17549435082228750797e-38f;
  const float xs = sub ? x * 8388608.0f : x;
  const uint32_t b = pp_f2u(xs);
  int e = (int)((b >> 23) & 0xffu) - 127 - (sub ? 23 : 0);
  float m = pp_u2f((b & 0x007fffffu) | 0x3f800000u);               /* [1, 2) */
  const int hi = m > 1.41421353816986083984375f;
  m = hi ? m * 0.5f : m;                                            /* [0.707, 1.414] */
  e += hi;
  const float lm = pp_log1p_red(m - 1.0f);
  const float ef = (float)e;
  const float lo = pp_fma(ef, 1.428606765330187045e-06f, lm);
  float y = pp_fma(ef, 0.693145751953125f, lo);
  y = (x == pp_u2f(0x7f800000u)) ? x : y;
  y = (x == 0.0f) ? pp_u2f(0xff800000u) : y;
  y = (x < 0.0f) ? pp_u2f(0x7fc00000u) : y;
  return (x != x) ? x : y;
}

/* log(x) for x in [2^-24, 1]: pp_logf without the special-case tests (same
 * arithmetic, so equal results on that domain). */
PPF_HD float pp_log_unit(float x) {
  const uint32_t b = pp_f2u(x);
  int e = (int)((b >> 23) & 0xffu) - 127;
  float m = pp_u2f((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421353816986083984375f) { m = m * 0.5f; e += 1; }
  const float lm = pp_log1p_red(m - 1.0f);
  const float ef = (float)e;
  const float lo = pp_fma(ef, 1.428606765330187045e-06f, lm);
  return pp_fma(ef, 0.693145751953125f, lo);
}

/* sin(2 pi u), cos(2 pi u) for u in [0, 1). */
PPF_HD void pp_sincos2pif(float u, float* sn, float* cs) {
  const float v = u * 4.0f;                 /* exact */
  const float qf = floorf(v);
  float r = v - qf;                         /* exact, [0,1) */
  const int q = ((int)qf) & 3;
  const int swap = r > 0.5f;
  if (swap) r = 1.0f - r;                   /* exact */
  const float t = r * 1.57079637050628662109375f;   /* pi/2 */
  const float t2 = t * t;
  float ps = -2.50521083854417188e-08f;     /* -1/11! */
  ps = pp_fma(ps, t2, 2.75573192239858907e-06f);   /* 1/9! */
  ps = pp_fma(ps, t2, -1.98412698412698413e-04f);  /* -1/7! */
  ps = pp_fma(ps, t2, 8.33333333333333333e-03f);   /* 1/5! */
  ps = pp_fma(ps, t2, -1.66666666666666667e-01f);  /* -1/3! */
  const float s = pp_fma(ps * t2, t, t);
  float pc = 2.08767569878680990e-09f;      /* 1/12! */
  pc = pp_fma(pc, t2, -2.75573192239858907e-07f);  /* -1/10! */
  pc = pp_fma(pc, t2, 2.48015873015873016e-05f);   /* 1/8! */
  pc = pp_fma(pc, t2, -1.38888888888888889e-03f);  /* -1/6! */
  pc = pp_fma(pc, t2, 4.16666666666666667e-02f);   /* 1/4! */
  pc = pp_fma(pc, t2, -0.5f);
  const float c = pp_fma(pc, t2, 1.0f);
  const float a = swap ? c : s;             /* sin of the in-quadrant angle */
  const float bb = swap ? s : c;            /* cos of the in-quadrant angle */
  /* rotate by q quarter turns: (a, bb) -> (bb, -a) -> (-a, -bb) -> (-bb, a) */
  const float s1 = (q & 1) ? bb : a;
  const float c1 = (q & 1) ? a : bb;
  *sn = (q >= 2) ? -s1 : s1;
  *cs = ((q == 1) | (q == 2)) ? -c1 : c1;
}

#endif /* PPF_DETMATH_H */
