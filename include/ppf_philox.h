/*
 * ppf_philox.h -- Philox4x32-10 counter-based generator and the draws built
 * on it, shared by the CUDA kernels and the C oracle.
 *
 * Philox4x32-10 is the published generator of Salmon, Moraes, Dror & Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3" (SC'11): multipliers
 * 0xD2511F53 / 0xCD9E8D57, Weyl key increments 0x9E3779B9 / 0xBB67AE85,
 * ten rounds.  Tests check it against the paper's known-answer vectors.
 *
 * Counter layout used by every kernel (one 64-bit key per filter):
 *   c0 = normal-stream block (normal i of a step comes from block i / 4)
 *   c1 = step s (0 = initial draw, i+1 = the step into observation i)
 *   c2 = purpose tag: 0 process noise, 1 resampling uniform (c0 = 0),
 *        2 IF2 parameter perturbation
 *   c3 = 0
 * Each call yields four 32-bit words; normals come in pairs by Box-Muller:
 *   u1 = ((w0 >> 8) + 1) 2^-24 in (0, 1],  u2 = (w1 >> 8) 2^-24 in [0, 1)
 *   z0 = sqrt(-2 log u1) cos(2 pi u2),     z1 = sqrt(-2 log u1) sin(2 pi u2)
 * with log / sin / cos from ppf_detmath.h, so draws are bit-identical on host
 * and device.
 */
#ifndef PPF_PHILOX_H
#define PPF_PHILOX_H

#include <stdint.h>
#include "ppf_detmath.h"

enum { PPF_TAG_PROCESS = 0, PPF_TAG_RESAMPLE = 1, PPF_TAG_PERTURB = 2 };

typedef struct { uint32_t v[4]; } pp_u32x4;

PPF_HD void pp_mulhilo(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
#if defined(__CUDA_ARCH__)
  *lo = a * b;
  *hi = __umulhi(a, b);
#else
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *lo = (uint32_t)p;
  *hi = (uint32_t)(p >> 32);
#endif
}

PPF_HD pp_u32x4 pp_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                 uint32_t k0, uint32_t k1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    pp_mulhilo(0xD2511F53u, c0, &hi0, &lo0);
    pp_mulhilo(0xCD9E8D57u, c2, &hi1, &lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  pp_u32x4 out;
  out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
  return out;
}

/* Box-Muller pair from two words. */
PPF_HD void pp_boxmuller(uint32_t wa, uint32_t wb, float* z0, float* z1) {
  const float u1 = (float)((wa >> 8) + 1u) * 5.9604644775390625e-08f;  /* 2^-24 */
  const float u2 = (float)(wb >> 8) * 5.9604644775390625e-08f;
  const float rr = sqrtf(-2.0f * pp_log_unit(u1));
  float s, c;
  pp_sincos2pif(u2, &s, &c);
  *z0 = rr * c;
  *z1 = rr * s;
}

#if defined(__CUDACC__)
/* Box-Muller pair from the same two words with the SFU approximations
 * (__log2f, rsqrtf, __sincosf; device only).  Used by the PPF_F_FAST kernels:
 * close to pp_boxmuller (a few ulp) but not bit-identical, and there is no
 * host counterpart.  sin / cos are taken at 2 pi (u2 - 1/2) in [-pi, pi),
 * where the approximations hold their accuracy, and negated. */
__device__ __forceinline__ void pp_boxmuller_fast(uint32_t wa, uint32_t wb, float* z0, float* z1) {
  const float u1 = (float)((wa >> 8) + 1u) * 5.9604644775390625e-08f;
  const float u2 = (float)(wb >> 8) * 5.9604644775390625e-08f;
  const float t = -1.3862943611198906f * __log2f(u1);       /* -2 ln u1 */
  const float rr = t > 0.0f ? t * rsqrtf(t) : 0.0f;
  float s, c;
  __sincosf(6.283185307179586f * (u2 - 0.5f), &s, &c);
  *z0 = -rr * c;
  *z1 = -rr * s;
}

__device__ __forceinline__ void pp_normal4_fast(uint64_t seed, uint32_t call, uint32_t s, uint32_t tag,
                                                float* z4) {
  const pp_u32x4 w = pp_philox4x32_10(call, s, tag, 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
  pp_boxmuller_fast(w.v[0], w.v[1], &z4[0], &z4[1]);
  pp_boxmuller_fast(w.v[2], w.v[3], &z4[2], &z4[3]);
}
#endif

/* Normal number i of the stream (step s, tag) of one filter:
 * element i % 4 of the four normals made from Philox(c0 = i / 4, s, tag, 0).
 * Particle k draws the n consecutive normals i = k n ... k n + n - 1, so a
 * group of 4 consecutive particles consumes exactly n Philox calls and 2n
 * Box-Muller pairs -- every word is used. */
PPF_HD void pp_normal4(uint64_t seed, uint32_t call, uint32_t s, uint32_t tag, float* z4) {
  const pp_u32x4 w = pp_philox4x32_10(call, s, tag, 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
  pp_boxmuller(w.v[0], w.v[1], &z4[0], &z4[1]);
  pp_boxmuller(w.v[2], w.v[3], &z4[2], &z4[3]);
}

/* The n normals of particle k (n <= 16), computed one at a time; bit-identical
 * to the grouped computation the kernels use. */
PPF_HD void pp_normals(uint64_t seed, uint32_t k, uint32_t s, uint32_t tag, int n, float* z) {
  uint32_t cached = 0xffffffffu;
  float z4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int r = 0; r < n; ++r) {
    const uint32_t i = k * (uint32_t)n + (uint32_t)r;
    if ((i >> 2) != cached) {
      cached = i >> 2;
      pp_normal4(seed, cached, s, tag, z4);
    }
    z[r] = z4[i & 3u];
  }
}

/* pp_normals evaluating only the Box-Muller pairs that particle k uses (a
 * Philox block serves 4 normals; with n = 1 or 2 the other pair belongs to a
 * neighbour).  Bit-identical to pp_normals: same words, same pair arithmetic. */
PPF_HD void pp_normals_own(uint64_t seed, uint32_t k, uint32_t s, uint32_t tag, int n, float* z) {
  uint32_t cblk = 0xffffffffu, cpair = 0xffffffffu;
  pp_u32x4 w = {{0u, 0u, 0u, 0u}};
  float p0 = 0.0f, p1 = 0.0f;
  for (int r = 0; r < n; ++r) {
    const uint32_t i = k * (uint32_t)n + (uint32_t)r;
    if ((i >> 2) != cblk) {
      cblk = i >> 2;
      w = pp_philox4x32_10(cblk, s, tag, 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
    }
    if ((i >> 1) != cpair) {
      cpair = i >> 1;
      const int hi = (int)(cpair & 1u);
      pp_boxmuller(hi ? w.v[2] : w.v[0], hi ? w.v[3] : w.v[1], &p0, &p1);
    }
    z[r] = (i & 1u) ? p1 : p0;
  }
}

/* Resampling uniform for step s as a 32-bit fraction (U = u32 * 2^-32). */
PPF_HD uint32_t pp_resample_u32(uint64_t seed, uint32_t s) {
  const pp_u32x4 w = pp_philox4x32_10(0u, s, PPF_TAG_RESAMPLE, 0u, (uint32_t)seed,
                                      (uint32_t)(seed >> 32));
  return (w.v[0] >> 8) << 8;   /* 24 significant bits, as a float uniform would carry */
}

/* Injected float uniform U in [0,1) to the 32-bit fraction: floor(U * 2^32). */
PPF_HD uint32_t pp_u32_from_float(float u) {
  if (!(u > 0.0f)) return 0u;
  if (u >= 1.0f) return 0xffffffffu;
  return (uint32_t)(u * 4294967296.0f);
}

#endif /* PPF_PHILOX_H */
