/*
 * ppf_sample.h -- measurement draws for simulation (rmeas), shared by the
 * CUDA kernels and the C oracle, bit-identical on both (same rules as
 * ppf_detmath.h: only correctly rounded IEEE operations, no contraction).
 *
 * Counter layout (extends ppf_philox.h, one 64-bit key per parameter set):
 *   tag 3, measurement normals: normal i of replicate k at step s comes from
 *          Philox(c0 = i / 4, s, 3, 0), numbered like the process normals
 *          (replicate k draws i = k n ... k n + n - 1);
 *   tag 4, count draws: replicate k at step s uses Philox(c0 = k, s, 4, c3 = i)
 *          for its i-th pair of tries (words 0, 1: first try; 2, 3: second).
 * Step s = t + 1 draws the observation y_t (s = 0 is the initial state).
 *
 * Poisson(lam):
 *   lam < 10   inversion: the CDF is summed from 0 with the float32 recurrence
 *              p_k = (p_{k-1} lam) / k until it exceeds one uniform u in [0, 1)
 *              (or stops growing in float32, or k reaches 64);
 *   lam >= 10  the transformed rejection method with squeeze (PTRS) of
 *              W. Hoermann, "The transformed rejection method for generating
 *              Poisson random variables", Insurance: Mathematics and Economics
 *              12 (1993) 39-45, with the paper's constants; log k! from a table
 *              below 16 and the Stirling series with three terms above.  At
 *              most 32 tries (acceptance is above 0.9 per try); after that
 *              rint(lam) is returned.
 *   lam == 0 gives 0, lam == +inf gives +inf, NaN or negative lam gives NaN.
 */
#ifndef PPF_SAMPLE_H
#define PPF_SAMPLE_H

#include <stdint.h>
#include "ppf_detmath.h"
#include "ppf_philox.h"

enum { PPF_TAG_MEASURE = 3, PPF_TAG_COUNT = 4 };

/* log k! for an integer-valued k >= 0. */
PPF_HD float pp_logfact(float k) {
  if (k < 16.0f) {
    switch ((int)k) {
      case 0: case 1: return 0.0f;
      case 2: return 0.693147180559945f;
      case 3: return 1.7917594692280554f;
      case 4: return 3.178053830347945f;
      case 5: return 4.787491742782047f;
      case 6: return 6.579251212010102f;
      case 7: return 8.525161361065415f;
      case 8: return 10.604602902745249f;
      case 9: return 12.801827480081467f;
      case 10: return 15.104412573075514f;
      case 11: return 17.502307845873887f;
      case 12: return 19.987214495661885f;
      case 13: return 22.55216385312342f;
      case 14: return 25.191221182738683f;
      default: return 27.89927138384089f;
    }
  }
  /* log Gamma(x), x = k + 1 >= 17: (x - 1/2) log x - x + log(2 pi)/2
   * + 1/(12 x) - 1/(360 x^3) + 1/(1260 x^5) */
  const float x = k + 1.0f;
  const float ix = 1.0f / x;
  const float ix2 = ix * ix;
  const float corr = ix * (0.0833333333333f - ix2 * (0.00277777777778f - ix2 * 0.000793650793651f));
  return (x - 0.5f) * pp_logf(x) - x + 0.918938533204672742f + corr;
}

/* One Poisson(lam) draw of replicate k at step s, as a float count. */
PPF_HD float pp_poisson(float lam, uint64_t seed, uint32_t k, uint32_t s) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  if (lam != lam || lam < 0.0f) return pp_u2f(0x7fc00000u);
  if (lam == 0.0f) return 0.0f;
  if (lam == pp_u2f(0x7f800000u)) return lam;
  if (lam < 10.0f) {
    const pp_u32x4 w = pp_philox4x32_10(k, s, PPF_TAG_COUNT, 0u, k0, k1);
    const float u = (float)(w.v[0] >> 8) * 5.9604644775390625e-08f;   /* [0, 1) */
    float p = pp_expf(-lam);
    float cdf = p;
    float n = 0.0f;
    for (int i = 0; i < 64 && u >= cdf; ++i) {
      n = n + 1.0f;
      p = (p * lam) / n;
      const float next = cdf + p;
      if (next == cdf) break;
      cdf = next;
    }
    return n;
  }
  const float smu = sqrtf(lam);
  const float b = 0.931f + 2.53f * smu;
  const float a = -0.059f + 0.02483f * b;
  const float inv_alpha = 1.1239f + 1.1328f / (b - 3.4f);
  const float vr = 0.9277f - 3.6224f / (b - 2.0f);
  const float loglam = pp_logf(lam);
  const float log_ia = pp_logf(inv_alpha);
  for (uint32_t i = 0; i < 16u; ++i) {
    const pp_u32x4 w = pp_philox4x32_10(k, s, PPF_TAG_COUNT, i, k0, k1);
    for (int h = 0; h < 2; ++h) {
      const float U = (float)(w.v[2 * h] >> 8) * 5.9604644775390625e-08f - 0.5f;        /* [-1/2, 1/2) */
      const float V = (float)((w.v[2 * h + 1] >> 8) + 1u) * 5.9604644775390625e-08f;   /* (0, 1] */
      const float us = 0.5f - fabsf(U);
      const float n = floorf((2.0f * a / us + b) * U + lam + 0.43f);
      if (us >= 0.07f && V <= vr) return n;
      if (n < 0.0f || (us < 0.013f && V > us)) continue;
      const float lhs = pp_logf(V) + log_ia - pp_logf(a / (us * us) + b);
      const float rhs = -lam + n * loglam - pp_logfact(n);
      if (lhs <= rhs) return n;
    }
  }
  return pp_rint(lam);
}

#endif /* PPF_SAMPLE_H */
