// ppf_core.cuh -- shared device primitives of the particle-filter kernels:
// ordered-float keys for atomic max/min, warp/block reductions and scans,
// the fixed-point weight, and the exact systematic-resampling offset.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "ppf.h"
#include "ppf_detmath.h"
#include "ppf_philox.h"

namespace ppf {

typedef unsigned __int128 u128;

constexpr float kQScale = 1099511627776.0f;        // 2^40, fixed-point weight scale
constexpr double kLn2 = 0.69314718055994530942;
constexpr long long kSpinCap = 1ll << 22;          // bounded waits: then PPF_ETIMEOUT
                                                   // (ppf_debug_set_wait_limit lowers it per call)

// Per-filter, per-step accumulators (double-buffered by step parity).
constexpr int kMaxDim = 9;                          // largest state dimension (LG 9 x 9)
struct Acc {
  unsigned int maxkey, minkey, nan, pad;
  double s2;              // sum e^2 (ESS)
  double fx[kMaxDim];     // sum x e (filter mean)
  double px[kMaxDim];     // sum x (prediction mean)
};
static_assert(sizeof(Acc) == 168, "Acc layout");

__device__ __forceinline__ unsigned int fkey(float f) {
  const unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float keyf(unsigned int k) {
  const unsigned int b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(b);
}

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Strong relaxed accesses at GPU scope (coherent through L2, no ordering of
// other memory): enough for a word that carries its own status and value.
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ---- TMA 1-D bulk copies (global -> this CTA's shared memory, no multicast)
// tracked by an mbarrier transaction count.  Addresses and sizes must be
// multiples of 16 bytes; waits are bounded.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Wait for phase `parity` of the barrier; false if the bounded wait gave up
// after `cap` polls (cap 0: gives up at once).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long cap = kSpinCap) {
  for (long long i = 0; i < cap; ++i) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---- grid-wide barrier for cooperative (co-resident) launches.  Three words
// in the workspace's zeroed control block: arrivals, generation, abort.  The
// last CTA to arrive resets the arrival count and advances the generation;
// the others poll the generation.  Every poll loop is bounded: a CTA that
// gives up sets error bit 1 (PPF_ETIMEOUT) and the abort word, so the other
// CTAs stop at their next barrier instead of waiting in turn, and the kernel
// ends.  Ordering: the CTA barrier orders every thread's writes before thread
// 0's acquire-release add of its arrival; the last arrival's add acquires
// all earlier ones and its release of the new generation is acquired by the
// waiting threads, and a CTA barrier then orders every thread's reads after
// it -- no sequentially consistent fence is needed.
struct GridBar {
  unsigned int* count;
  unsigned int* gen;
  unsigned int* abort;
  uint32_t* err;
  unsigned int n;       // CTAs in the grid
  long long cap;        // polls before giving up
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u32(unsigned int* p, unsigned int v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// acquire + release: the last CTA to arrive also acquires the earlier
// arrivals' writes (their release-adds form one release sequence on `count`).
__device__ __forceinline__ unsigned int atom_add_acq_rel_u32(unsigned int* p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Returns false when the barrier gave up (this CTA's or another's wait).
__device__ __forceinline__ bool grid_sync(const GridBar& g) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int gen = ld_relaxed_u32(g.gen);   // cannot advance before this CTA arrives
    if (atom_add_acq_rel_u32(g.count, 1u) == g.n - 1) {
      st_relaxed_u32(g.count, 0u);
      st_release_u32(g.gen, gen + 1);
    } else {
      long long i = 0;
      while (ld_acquire_u32(g.gen) == gen) {
        if (++i > g.cap || ld_relaxed_u32(g.abort) != 0u) { ok = 0; break; }
        __nanosleep(20);
      }
    }
    if (!ok) {
      atomicOr(g.err, 1u);
      atomicExch(g.abort, 1u);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Counting form: every CTA adds 1 to `count` (release) per barrier and waits
// (acquire) until it reaches epoch * n for its own barrier number `epoch`
// (1, 2, ...; the count starts at 0 and only grows).  No CTA resets or
// advances anything, so a barrier costs one fire-and-forget add and the
// polls: one round trip less than the arrival-then-generation form.  The same
// bounded wait, error and abort words as grid_sync.
__device__ __forceinline__ bool grid_sync_count(const GridBar& g, unsigned int epoch) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(g.count) : "memory");
    const unsigned int target = epoch * g.n;
    long long i = 0;
    while ((int)(ld_acquire_u32(g.count) - target) < 0) {
      if (++i > g.cap || ld_relaxed_u32(g.abort) != 0u) { ok = 0; break; }
      __nanosleep(20);
    }
    if (!ok) {
      atomicOr(g.err, 1u);
      atomicExch(g.abort, 1u);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// The fixed-point weight q = rint(exp(w - M) * 2^40) (collapsed filters: 1),
// in two halves: the float e = qweight_e(w, M, collapsed) and
// q = qweight_from_e(e).  On a resampling step the streaming path's k_sum
// stores e over the parent log-weight, which nothing else reads afterwards,
// and k_resprop forms q from it without repeating the exp.  e * 2^40 is exact
// (e <= 1), so q is the same either way.
__device__ __forceinline__ float qweight_e(float w, float M, bool collapsed) {
  if (collapsed) return 9.094947017729282e-13f;   // 2^-40: q = 1
  if (w != w) return 0.0f;
  return pp_expq(w - M);     // equals pp_expf(w - M) wherever the quantised value can be >= 1
}
__device__ __forceinline__ uint64_t qweight_from_e(float e) { return __float2ull_rn(e * kQScale); }
// qweight_e with the SFU exponential (PPF_F_FAST): e in (0, 1], not bit-identical.
template <bool FAST>
__device__ __forceinline__ float qweight_e_t(float w, float M, bool collapsed) {
  if (!FAST) return qweight_e(w, M, collapsed);
  if (collapsed) return 9.094947017729282e-13f;
  if (w != w) return 0.0f;
  return __expf(w - M);
}
__device__ __forceinline__ uint64_t qweight(float w, float M, bool collapsed) {
  return qweight_from_e(qweight_e(w, M, collapsed));
}

// Number of systematic points strictly below the CDF value C:
//   nchild(C) = #{ k in [0,J) : (u32 + k 2^32) * tot < C * J * 2^32 }.
// A double-precision estimate is corrected with exact 128-bit comparisons.
__device__ __forceinline__ int nchild(uint64_t C, uint64_t tot, uint32_t u32, int J) {
  const u128 L = (u128)C * (u128)((uint64_t)J << 32);
  const u128 ut = (u128)u32 * (u128)tot;
  if (L <= ut) return 0;
  const double est = (double)C * (double)J / (double)tot - (double)u32 * 2.3283064365386963e-10;
  long long k = (long long)ceil(est);
  if (k < 0) k = 0;
  if (k > J) k = J;
  const u128 step = (u128)tot << 32;
  // invariant wanted: R(k-1) < L <= R(k), R(k) = ut + k*step
  while (k > 0 && ut + (u128)(k - 1) * step >= L) --k;
  while (k < J && ut + (u128)k * step < L) ++k;
  return (int)k;
}

// ------------------------------- warp / block ------------------------------

__device__ __forceinline__ uint64_t warp_incl_scan_u64(uint64_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned int warp_max_u32(unsigned int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ unsigned int warp_min_u32(unsigned int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_incl_max_i32(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = max(v, n);
  }
  return v;
}

// Block exclusive scan of one uint64 per thread; returns the exclusive prefix
// and writes the block total.  `sm` needs TPB/32 + 1 entries.
template <int TPB>
__device__ __forceinline__ uint64_t block_excl_scan_u64(uint64_t v, uint64_t* sm, uint64_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = TPB / 32;
  const uint64_t inc = warp_incl_scan_u64(v);
  if (lane == 31) sm[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint64_t wv = lane < NW ? sm[lane] : 0ull;
    const uint64_t wi = warp_incl_scan_u64(wv);
    if (lane < NW) sm[lane] = wi - wv;
    if (lane == NW - 1) sm[NW] = wi;
  }
  __syncthreads();
  const uint64_t res = sm[warp] + inc - v;
  total = sm[NW];
  __syncthreads();
  return res;
}

// block_excl_scan_u64 with one barrier: warp scans, then every thread adds the
// totals of the warps before its own.  The caller must not write `sm` again
// before another barrier.
template <int TPB>
__device__ __forceinline__ uint64_t block_excl_scan_u64_1b(uint64_t v, uint64_t* sm, uint64_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t inc = warp_incl_scan_u64(v);
  if (lane == 31) sm[warp] = inc;
  __syncthreads();
  uint64_t before = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < TPB / 32; ++w) {
    const uint64_t x = sm[w];
    before += (w < warp) ? x : 0ull;
    tot += x;
  }
  total = tot;
  return before + inc - v;
}

// Block exclusive max-scan of one int per thread (identity -1).
template <int TPB>
__device__ __forceinline__ int block_excl_max_i32(int v, int* sm, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = TPB / 32;
  const int inc = warp_incl_max_i32(v);
  int exc = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) exc = -1;
  if (lane == 31) sm[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int wv = lane < NW ? sm[lane] : -1;
    const int wi = warp_incl_max_i32(wv);
    int we = __shfl_up_sync(0xffffffffu, wi, 1);
    if (lane == 0) we = -1;
    if (lane < NW) sm[lane] = we;
    if (lane == NW - 1) sm[NW] = wi;
  }
  __syncthreads();
  const int res = max(sm[warp], exc);
  total = sm[NW];
  __syncthreads();
  return res;
}

template <int TPB>
__device__ __forceinline__ double block_sum_f64(double v, double* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = TPB / 32;
  v = warp_sum_f64(v);
  if (lane == 0) sm[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < NW ? sm[lane] : 0.0;
    r = warp_sum_f64(r);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

template <int TPB>
__device__ __forceinline__ void block_maxmin_u32(unsigned int& mx, unsigned int& mn, unsigned int* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = TPB / 32;
  mx = warp_max_u32(mx);
  mn = warp_min_u32(mn);
  if (lane == 0) { sm[warp] = mx; sm[NW + warp] = mn; }
  __syncthreads();
  if (warp == 0) {
    unsigned int a = lane < NW ? sm[lane] : 0u;
    unsigned int b = lane < NW ? sm[NW + lane] : 0xffffffffu;
    a = warp_max_u32(a);
    b = warp_min_u32(b);
    mx = a; mn = b;
  }
  __syncthreads();
}

}  // namespace ppf
